// dimgpu_slabs.cu — one DIM grid decomposed into slabs along its slowest
// axis, one slab per GPU (include/dimgpu.h: dimgpu_slabs_*).  The B200
// counterpart of the reference's slab-decomposed MPI driver
// (src/app/dim_mpi_main.cpp:116-124 slabs, :383-423 halo exchange, :758 the
// dt reduction), in one process that drives every GPU through its own stream.
//
// Slab k owns planes [z0_k, z1_k) of the split axis and holds a session of
// the extended range [z0_k - 3, z1_k + 3) (clipped at the grid's ends): the
// split sweep of an owned cell reads U[i-3 .. i+3] along the line (and the
// line-end rules act on the extended ends, three cells away from every owned
// cell), so three ghost planes make every owned cell's update bit-identical
// to the single-grid step.  (The reference exchanges two, which is why its
// MPI run is not bit-identical to its serial one.)  A step:
//
//   CFL      each slab reduces its owned cells on its device; the host takes
//            min(dt_max, minimum over slabs), the same value as one grid's;
//   sweeps   per axis in x, y, z order; before the sweep along the split
//            axis, every slab's ghost planes are refreshed from its
//            neighbours' owned planes (device-to-device or peer copies, one
//            per component and side, ordered by events: the copies wait for
//            the neighbour's previous fill, the neighbour waits for the
//            copies before it writes that buffer again);
//   fill     the boundary fill of every slab's extended range: at the
//            grid's ends it is the real fill; at an internal cut it writes
//            ghost planes only, which the next exchange overwrites.
//
// The slabs may share a device (then the exchange is a plain device copy):
// that is how the decomposition is tested on one GPU against a single
// session, bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dimgpu_session.h"

using namespace dimgpu;

namespace {

constexpr int kGhost = 3;

struct Slab {
    int device = 0;
    int own0 = 0, own1 = 0;   // owned planes [own0, own1) of the split axis
    int ext0 = 0, ext1 = 0;   // planes held by the session
    dimgpu_session* s = nullptr;
    cudaEvent_t filled = nullptr;   // after the last boundary fill
    cudaEvent_t copied = nullptr;   // after the copies into this slab's ghosts
    double* dt_host = nullptr;      // pinned
};

}  // namespace

struct dimgpu_slabs {
    dimgpu_desc desc{};
    int axis = 0;
    long long plane = 0;   // cells per plane of the split axis
    int V = 0;
    std::vector<Slab> slabs;
    std::string msg;
};

namespace {

int lfail(dimgpu_slabs* L, int code, const std::string& m)
{
    if (L) L->msg = m;
    set_sessionless_error(m);
    return code;
}

int lcuda(dimgpu_slabs* L, cudaError_t e, const char* what)
{
    return lfail(L, e == cudaErrorMemoryAllocation ? DIMGPU_E_OOM : DIMGPU_E_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

void destroy_slabs(dimgpu_slabs* L)
{
    for (auto& sl : L->slabs) {
        if (sl.s) {
            cudaSetDevice(sl.device);
            dimgpu_destroy(sl.s);
        }
        if (sl.filled) cudaEventDestroy(sl.filled);
        if (sl.copied) cudaEventDestroy(sl.copied);
        if (sl.dt_host) cudaFreeHost(sl.dt_host);
    }
    delete L;
}

// Copy planes [p0, p1) (global plane numbers) of every component from slab
// `src`'s current buffer into slab `dst`'s current buffer, on dst's stream.
cudaError_t copy_planes(dimgpu_slabs* L, Slab& src, Slab& dst, int p0, int p1)
{
    if (p1 <= p0) return cudaSuccess;
    const size_t bytes = sizeof(double) * (size_t)(p1 - p0) * (size_t)L->plane;
    const long long src_n = (long long)(src.ext1 - src.ext0) * L->plane;
    const long long dst_n = (long long)(dst.ext1 - dst.ext0) * L->plane;
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < L->V && e == cudaSuccess; ++c) {
        const double* from = src.s->buf[src.s->cur] + (size_t)c * src_n + (size_t)(p0 - src.ext0) * L->plane;
        double* to = dst.s->buf[dst.s->cur] + (size_t)c * dst_n + (size_t)(p0 - dst.ext0) * L->plane;
        if (src.device == dst.device)
            e = cudaMemcpyAsync(to, from, bytes, cudaMemcpyDeviceToDevice, dst.s->stream);
        else
            e = cudaMemcpyPeerAsync(to, dst.device, from, src.device, bytes, dst.s->stream);
    }
    return e;
}

// Refresh every slab's ghost planes from its neighbours' owned planes.
cudaError_t exchange(dimgpu_slabs* L)
{
    const int n = (int)L->slabs.size();
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        Slab& sl = L->slabs[(size_t)k];
        cudaSetDevice(sl.device);
        e = cudaEventRecord(sl.filled, sl.s->stream);
    }
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        Slab& dst = L->slabs[(size_t)k];
        cudaSetDevice(dst.device);
        if (k > 0) {
            Slab& lo = L->slabs[(size_t)k - 1];
            e = cudaStreamWaitEvent(dst.s->stream, lo.filled, 0);
            if (e == cudaSuccess) e = copy_planes(L, lo, dst, dst.ext0, dst.own0);
        }
        if (e == cudaSuccess && k + 1 < n) {
            Slab& hi = L->slabs[(size_t)k + 1];
            e = cudaStreamWaitEvent(dst.s->stream, hi.filled, 0);
            if (e == cudaSuccess) e = copy_planes(L, hi, dst, dst.own1, dst.ext1);
        }
        if (e == cudaSuccess) e = cudaEventRecord(dst.copied, dst.s->stream);
    }
    // a slab writes the buffer its neighbours read from only after their copies
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        Slab& sl = L->slabs[(size_t)k];
        cudaSetDevice(sl.device);
        if (k > 0) e = cudaStreamWaitEvent(sl.s->stream, L->slabs[(size_t)k - 1].copied, 0);
        if (e == cudaSuccess && k + 1 < n) e = cudaStreamWaitEvent(sl.s->stream, L->slabs[(size_t)k + 1].copied, 0);
    }
    return e;
}

}  // namespace

extern "C" {

int dimgpu_slabs_create(const dimgpu_desc* desc, int nslabs, const int* devices, dimgpu_slabs** out)
{
    if (!desc || !out || nslabs < 1) return lfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_slabs_create: bad argument");
    *out = nullptr;
    if (desc->model != DIMGPU_MODEL_DIM || desc->time_update != DIMGPU_TIME_SPLIT)
        return lfail(nullptr, DIMGPU_E_UNSUPPORTED, "dimgpu_slabs_create: the split DIM step only");
    if (desc->dim < 2) return lfail(nullptr, DIMGPU_E_UNSUPPORTED, "dimgpu_slabs_create: 2D and 3D grids only");
    const int axis = desc->dim - 1;
    const int N = desc->N[axis];
    if (N / nslabs < kGhost)
        return lfail(nullptr, DIMGPU_E_INVALID_ARG,
                     "dimgpu_slabs_create: every slab needs at least 3 planes of the split axis");
    auto* L = new dimgpu_slabs();
    L->desc = *desc;
    L->axis = axis;
    L->V = 2 * desc->nmat + desc->dim;
    L->plane = 1;
    for (int a = 0; a < axis; ++a) L->plane *= desc->N[a];
    int prev = 0;
    cudaSetDevice(devices ? devices[0] : 0);
    for (int k = 0; k < nslabs; ++k) {
        Slab sl;
        sl.device = devices ? devices[k] : 0;
        sl.own0 = prev;
        sl.own1 = (int)((long long)N * (k + 1) / nslabs);
        prev = sl.own1;
        sl.ext0 = std::max(0, sl.own0 - kGhost);
        sl.ext1 = std::min(N, sl.own1 + kGhost);
        L->slabs.push_back(sl);
    }
    for (auto& sl : L->slabs) {
        cudaError_t e = cudaSetDevice(sl.device);
        if (e != cudaSuccess) {
            const int rc = lcuda(L, e, "dimgpu_slabs_create");
            destroy_slabs(L);
            return rc;
        }
        dimgpu_desc d = *desc;
        d.N[axis] = sl.ext1 - sl.ext0;
        int rc = dimgpu_create(&d, &sl.s);
        if (rc != DIMGPU_OK) {
            const std::string m = dimgpu_last_error(nullptr);
            destroy_slabs(L);
            return lfail(nullptr, rc, "dimgpu_slabs_create: " + m);
        }
        e = cudaEventCreateWithFlags(&sl.filled, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.dt_host, sizeof(double));
        if (e != cudaSuccess) {
            const int rc2 = lcuda(L, e, "dimgpu_slabs_create");
            destroy_slabs(L);
            return rc2;
        }
    }
    // peer access between distinct devices where the platform allows it
    for (auto& a : L->slabs)
        for (auto& b : L->slabs) {
            if (a.device == b.device) continue;
            int can = 0;
            cudaDeviceCanAccessPeer(&can, a.device, b.device);
            if (can) {
                cudaSetDevice(a.device);
                cudaDeviceEnablePeerAccess(b.device, 0);
                cudaGetLastError();  // already enabled is fine
            }
        }
    *out = L;
    return DIMGPU_OK;
}

int dimgpu_slabs_destroy(dimgpu_slabs* L)
{
    if (L) destroy_slabs(L);
    return DIMGPU_OK;
}

const char* dimgpu_slabs_last_error(const dimgpu_slabs* L) { return L ? L->msg.c_str() : ""; }

int dimgpu_slabs_upload(dimgpu_slabs* L, const double* soa, size_t count)
{
    if (!L || !soa) return lfail(L, DIMGPU_E_INVALID_ARG, "dimgpu_slabs_upload: null argument");
    const long long ncell = L->plane * L->desc.N[L->axis];
    if (count != (size_t)L->V * (size_t)ncell) return lfail(L, DIMGPU_E_INVALID_ARG, "dimgpu_slabs_upload: size mismatch");
    for (auto& sl : L->slabs) {
        cudaSetDevice(sl.device);
        const long long n = (long long)(sl.ext1 - sl.ext0) * L->plane;
        cudaError_t e = cudaSuccess;
        for (int c = 0; c < L->V && e == cudaSuccess; ++c)
            e = cudaMemcpyAsync(sl.s->buf[sl.s->cur] + (size_t)c * n, soa + (size_t)c * ncell + (size_t)sl.ext0 * L->plane,
                                sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, sl.s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sl.s->stream);
        if (e != cudaSuccess) return lcuda(L, e, "dimgpu_slabs_upload");
    }
    return DIMGPU_OK;
}

int dimgpu_slabs_download(dimgpu_slabs* L, double* soa, size_t count)
{
    if (!L || !soa) return lfail(L, DIMGPU_E_INVALID_ARG, "dimgpu_slabs_download: null argument");
    const long long ncell = L->plane * L->desc.N[L->axis];
    if (count != (size_t)L->V * (size_t)ncell)
        return lfail(L, DIMGPU_E_INVALID_ARG, "dimgpu_slabs_download: size mismatch");
    for (auto& sl : L->slabs) {
        cudaSetDevice(sl.device);
        const long long n = (long long)(sl.ext1 - sl.ext0) * L->plane;
        const long long owned = (long long)(sl.own1 - sl.own0) * L->plane;
        cudaError_t e = cudaSuccess;
        for (int c = 0; c < L->V && e == cudaSuccess; ++c)
            e = cudaMemcpyAsync(soa + (size_t)c * ncell + (size_t)sl.own0 * L->plane,
                                sl.s->buf[sl.s->cur] + (size_t)c * n + (size_t)(sl.own0 - sl.ext0) * L->plane,
                                sizeof(double) * (size_t)owned, cudaMemcpyDeviceToHost, sl.s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sl.s->stream);
        if (e != cudaSuccess) return lcuda(L, e, "dimgpu_slabs_download");
    }
    return DIMGPU_OK;
}

int dimgpu_slabs_step(dimgpu_slabs* L, double cfl, double dt_max, double* dt_out)
{
    if (!L) return lfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_slabs_step: null argument");
    if (!(cfl > 0.0)) return lfail(L, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: cfl must be positive");
    if (!(dt_max > 0.0)) return lfail(L, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: dt_max must be positive");
    cudaError_t e = cudaSuccess;
    // CFL over every slab's owned cells, reduced on the host
    for (auto& sl : L->slabs) {
        cudaSetDevice(sl.device);
        const long long b = (long long)(sl.own0 - sl.ext0) * L->plane;
        const long long en = (long long)(sl.own1 - sl.ext0) * L->plane;
        e = session_cfl_range(sl.s, cfl, dt_max, b, en);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.dt_host, sl.s->dt, sizeof(double), cudaMemcpyDeviceToHost, sl.s->stream);
        if (e != cudaSuccess) return lcuda(L, e, "dimgpu_slabs_step");
    }
    double dt = dt_max;
    for (auto& sl : L->slabs) {
        cudaSetDevice(sl.device);
        e = cudaStreamSynchronize(sl.s->stream);
        if (e != cudaSuccess) return lcuda(L, e, "dimgpu_slabs_step");
        dt = std::min(dt, *sl.dt_host);  // std::min(dt, candidate), as compute_dt_cfl reduces
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) return lfail(L, DIMGPU_E_NONFINITE, "run_dim_case: non-positive timestep");
    // the common dt into every slab's device copy (from pinned memory: the
    // host writes dt_host again only after the next CFL copy has landed)
    for (auto& sl : L->slabs) {
        cudaSetDevice(sl.device);
        *sl.dt_host = dt;
        e = cudaMemcpyAsync(sl.s->dt, sl.dt_host, sizeof(double), cudaMemcpyHostToDevice, sl.s->stream);
        if (e != cudaSuccess) return lcuda(L, e, "dimgpu_slabs_step");
    }
    for (int dir = 0; dir < L->desc.dim && e == cudaSuccess; ++dir) {
        if (dir == L->axis && L->slabs.size() > 1) e = exchange(L);
        for (auto& sl : L->slabs) {
            if (e != cudaSuccess) break;
            cudaSetDevice(sl.device);
            e = session_sweep(sl.s, dir);
            if (e == cudaSuccess) e = session_bc(sl.s);
        }
    }
    if (e != cudaSuccess) return lcuda(L, e, "dimgpu_slabs_step");
    for (auto& sl : L->slabs) {
        cudaSetDevice(sl.device);
        const int rc = session_check(sl.s);
        if (rc != DIMGPU_OK) return lfail(L, rc, dimgpu_last_error(sl.s));
    }
    if (dt_out) *dt_out = dt;
    return DIMGPU_OK;
}

}  // extern "C"
