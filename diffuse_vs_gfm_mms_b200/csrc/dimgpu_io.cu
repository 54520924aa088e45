// dimgpu_io.cu — initial fields generated on the device and the asynchronous
// CSV writer of a session's state (include/dimgpu.h: dimgpu_init_*,
// dimgpu_csv_*).
//
// The CSV writer keeps the reference's format byte for byte
// (dim::write_csv, src/io/dim_write_csv.hpp:15-125): the same header, one row
// per cell in linear (x-fastest) order, every value printed as std::ostream
// prints a double by default — "%.6g".  The per-cell values come from the
// device (dim_io.cuh: csv_records_kernel, the step's own bit-faithful
// cons_to_prim), in chunks through two pinned host buffers, and host threads
// format each chunk's rows in parallel and append them in order.  The state is
// first copied into a snapshot buffer on the device, so the session may keep
// stepping while the file is written.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "dim_io.cuh"
#include "dimgpu_session.h"

using namespace dimgpu;

namespace {

constexpr long long kCsvChunk = 1 << 20;  // cells per device -> host chunk

template<int NM, int D>
cudaError_t launch_csv_records(const double* st, const Grid& g, const Mats& M, const CsvGeom& geo, long long c0,
                               long long n, double* rec, cudaStream_t s)
{
    const long long blocks = (n + 255) / 256;
    csv_records_kernel<NM, D><<<(unsigned)blocks, 256, 0, s>>>(st, g, M, geo, c0, n, rec);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t csv_records(int nm, int dim, const double* st, const Grid& g, const Mats& M, const CsvGeom& geo,
                        long long c0, long long n, double* rec, cudaStream_t s)
{
    switch (nm * 10 + dim) {
#define CSV_CASE(NM, D) \
        case NM * 10 + D: return launch_csv_records<NM, D>(st, g, M, geo, c0, n, rec, s);
        CSV_CASE(1, 1) CSV_CASE(1, 2) CSV_CASE(1, 3)
        CSV_CASE(2, 1) CSV_CASE(2, 2) CSV_CASE(2, 3)
        CSV_CASE(3, 1) CSV_CASE(3, 2) CSV_CASE(3, 3)
        CSV_CASE(4, 1) CSV_CASE(4, 2) CSV_CASE(4, 3)
#undef CSV_CASE
        default: return cudaErrorInvalidValue;
    }
}

// Appends the row of one record.  The reference writes the coordinates, rho
// and the velocities each followed by ",", then "p,e", then ",value" per
// fraction, material density and mass: one "," between consecutive values.
void format_row(const double* r, int R, std::string& out)
{
    char buf[32];
    for (int q = 0; q < R; ++q) {
        const int len = std::snprintf(buf, sizeof buf, "%.6g", r[q]);
        out.append(buf, (size_t)len);
        out.push_back(q + 1 < R ? ',' : '\n');
    }
}

std::string csv_header(int nmat, int dim)
{
    std::string h;
    for (int d = 0; d < dim; ++d) h += "x" + std::to_string(d) + ",";
    h += "rho,";
    for (int d = 0; d < dim; ++d) h += "u" + std::to_string(d) + ",";
    h += "p,e";
    for (int k = 0; k < nmat; ++k) h += ",alpha" + std::to_string(k);
    for (int k = 0; k < nmat; ++k) h += ",rho_mat" + std::to_string(k);
    for (int k = 0; k < nmat; ++k) h += ",mass" + std::to_string(k);
    h += "\n";
    return h;
}

}  // namespace

struct dimgpu_csv_writer {
    std::string filename;
    int nmat = 0, dim = 0, R = 0, threads = 1;
    long long ncell = 0;
    Grid g{};
    Mats M{};
    CsvGeom geo{};
    double* snapshot = nullptr;    // device copy of the state
    double* rec_dev[2] = {nullptr, nullptr};
    double* rec_host[2] = {nullptr, nullptr};  // pinned
    cudaStream_t stream = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    std::thread worker;
    int status = DIMGPU_OK;
    std::string msg;
};

namespace {

void csv_release(dimgpu_csv_writer* w)
{
    if (w->stream) cudaStreamSynchronize(w->stream);
    cudaFree(w->snapshot);
    for (int b = 0; b < 2; ++b) {
        cudaFree(w->rec_dev[b]);
        cudaFreeHost(w->rec_host[b]);
        if (w->done[b]) cudaEventDestroy(w->done[b]);
        w->rec_dev[b] = w->rec_host[b] = nullptr;
        w->done[b] = nullptr;
    }
    if (w->stream) cudaStreamDestroy(w->stream);
    w->snapshot = nullptr;
    w->stream = nullptr;
}

// The host side of the writer: chunk k's records are computed into rec_dev[k%2]
// and copied to rec_host[k%2] while chunk k-1 is being formatted.
void csv_run(dimgpu_csv_writer* w)
{
    FILE* f = std::fopen(w->filename.c_str(), "wb");
    if (!f) {
        w->status = DIMGPU_E_INVALID_ARG;
        w->msg = "dim::write_csv: failed to open file";
        return;
    }
    const std::string header = csv_header(w->nmat, w->dim);
    std::fwrite(header.data(), 1, header.size(), f);
    const long long nchunks = (w->ncell + kCsvChunk - 1) / kCsvChunk;
    auto enqueue = [&](long long k) -> cudaError_t {
        const int b = (int)(k & 1);
        const long long c0 = k * kCsvChunk;
        const long long n = std::min(kCsvChunk, w->ncell - c0);
        cudaError_t e = csv_records(w->nmat, w->dim, w->snapshot, w->g, w->M, w->geo, c0, n, w->rec_dev[b], w->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(w->rec_host[b], w->rec_dev[b], sizeof(double) * (size_t)(n * w->R),
                                cudaMemcpyDeviceToHost, w->stream);
        if (e == cudaSuccess) e = cudaEventRecord(w->done[b], w->stream);
        return e;
    };
    cudaError_t e = nchunks > 0 ? enqueue(0) : cudaSuccess;
    std::vector<std::string> parts((size_t)w->threads);
    for (long long k = 0; k < nchunks && e == cudaSuccess; ++k) {
        const int b = (int)(k & 1);
        e = cudaEventSynchronize(w->done[b]);
        if (e == cudaSuccess && k + 1 < nchunks) e = enqueue(k + 1);
        if (e != cudaSuccess) break;
        const long long n = std::min(kCsvChunk, w->ncell - k * kCsvChunk);
        const double* rec = w->rec_host[b];
        const int T = (int)std::min<long long>(w->threads, std::max<long long>(1, n / 4096));
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t) {
            pool.emplace_back([&, t]() {
                const long long lo = n * t / T, hi = n * (t + 1) / T;
                std::string& out = parts[(size_t)t];
                out.clear();
                out.reserve((size_t)(hi - lo) * (size_t)w->R * 13);
                for (long long i = lo; i < hi; ++i) format_row(rec + i * w->R, w->R, out);
            });
        }
        for (auto& th : pool) th.join();
        for (int t = 0; t < T; ++t) std::fwrite(parts[(size_t)t].data(), 1, parts[(size_t)t].size(), f);
    }
    if (std::fclose(f) != 0 && w->status == DIMGPU_OK) {
        w->status = DIMGPU_E_INVALID_ARG;
        w->msg = "dim::write_csv: failed to write file";
    }
    if (e != cudaSuccess) {
        w->status = DIMGPU_E_CUDA;
        w->msg = std::string("dimgpu_csv_write_async: ") + cudaGetErrorString(e);
    }
}

}  // namespace

extern "C" {

int dimgpu_csv_write_async(dimgpu_session* s, const char* filename, const double* domain_min,
                           const double* domain_max, int threads, dimgpu_csv_writer** out)
{
    if (!s || !filename || !domain_min || !domain_max || !out)
        return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_csv_write_async: null argument");
    if (s->desc.model != DIMGPU_MODEL_DIM)
        return session_fail(s, DIMGPU_E_UNSUPPORTED, "dimgpu_csv_write_async: the DIM model's writer only");
    *out = nullptr;
    auto w = std::make_unique<dimgpu_csv_writer>();
    w->filename = filename;
    w->nmat = s->desc.nmat;
    w->dim = s->desc.dim;
    w->R = csv_record_width(w->nmat, w->dim);
    w->ncell = s->ncell;
    w->g = s->g;
    w->M = s->M;
    const unsigned hw = std::thread::hardware_concurrency();
    w->threads = threads > 0 ? threads : (int)std::max(1u, hw);
    for (int d = 0; d < 3; ++d) {
        w->geo.xmin[d] = d < w->dim ? domain_min[d] : 0.0;
        // dx = (domain_max - domain_min) / N (write_csv, dim_write_csv.hpp:31-34)
        w->geo.dx[d] = d < w->dim ? (domain_max[d] - domain_min[d]) / (double)s->desc.N[d] : 0.0;
    }
    const size_t state_bytes = sizeof(double) * (size_t)s->V * (size_t)s->ncell;
    const long long chunk = std::min<long long>(kCsvChunk, std::max<long long>(s->ncell, 1));
    const size_t rec_bytes = sizeof(double) * (size_t)(chunk * w->R);
    cudaError_t e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&w->snapshot, state_bytes);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMalloc(&w->rec_dev[b], rec_bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&w->rec_host[b], rec_bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->done[b], cudaEventDisableTiming);
    }
    // Snapshot: the writer's stream waits for the session's pending work, copies
    // the state, and the session's later work waits for that copy.
    cudaEvent_t ready = nullptr, taken = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&taken, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w->stream, ready, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(w->snapshot, s->buf[s->cur], state_bytes, cudaMemcpyDeviceToDevice, w->stream);
    if (e == cudaSuccess) e = cudaEventRecord(taken, w->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->stream, taken, 0);
    if (ready) cudaEventDestroy(ready);
    if (taken) cudaEventDestroy(taken);
    if (e != cudaSuccess) {
        csv_release(w.get());
        return session_cuda_fail(s, e, "dimgpu_csv_write_async");
    }
    dimgpu_csv_writer* raw = w.release();
    raw->worker = std::thread(csv_run, raw);
    *out = raw;
    return DIMGPU_OK;
}

int dimgpu_csv_wait(dimgpu_csv_writer* w)
{
    if (!w) {
        set_sessionless_error("dimgpu_csv_wait: null writer");
        return DIMGPU_E_INVALID_ARG;
    }
    if (w->worker.joinable()) w->worker.join();
    csv_release(w);
    const int rc = w->status;
    if (rc != DIMGPU_OK) set_sessionless_error(w->msg);
    delete w;
    return rc;
}

int dimgpu_init_shock_bubble(dimgpu_session* s, const dimgpu_ic_shock_bubble* p)
{
    if (!s || !p) return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_init_shock_bubble: null argument");
    if (s->desc.model != DIMGPU_MODEL_DIM || s->desc.nmat != 2 || s->desc.dim != 2)
        return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_init_shock_bubble: needs a 2D two-material DIM session");
    if (!(p->thickness > 0.0))
        return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_init_shock_bubble: thickness must be positive");
    ShockBubbleIC ic;
    ic.cx = p->center[0];
    ic.cy = p->center[1];
    ic.radius = p->radius;
    ic.thickness = p->thickness;
    ic.sharpness = p->sharpness;
    ic.shock_x = p->shock_x;
    ic.zero_below = p->zero_below;
    ic.rho_post = p->rho_post;
    ic.u_post = p->u_post;
    ic.p_post = p->p_post;
    ic.rho_pre = p->rho_pre;
    ic.p_pre = p->p_pre;
    ic.rho_bubble = p->rho_bubble;
    ic.p_bubble = p->p_bubble;
    const long long blocks = (s->ncell + 255) / 256;
    ic_shock_bubble_kernel<<<(unsigned)blocks, 256, 0, s->stream>>>(s->buf[s->cur], s->g, s->M, ic);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? DIMGPU_OK : session_cuda_fail(s, e, "dimgpu_init_shock_bubble");
}

int dimgpu_init_bubble_cloud(dimgpu_session* s, const dimgpu_ic_bubble_cloud* p, const dimgpu_ic_bubble* bubbles,
                             int nbubbles)
{
    if (!s || !p || (nbubbles > 0 && !bubbles))
        return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_init_bubble_cloud: null argument");
    if (s->desc.model != DIMGPU_MODEL_DIM || s->desc.nmat != 2 || s->desc.dim != 3)
        return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_init_bubble_cloud: needs a 3D two-material DIM session");
    if (nbubbles < 0 || !(p->thickness > 0.0))
        return session_fail(s, DIMGPU_E_INVALID_ARG, "dimgpu_init_bubble_cloud: bad bubble count or thickness");
    std::vector<BubbleIC> hb((size_t)std::max(nbubbles, 1));
    for (int b = 0; b < nbubbles; ++b) {
        for (int a = 0; a < 3; ++a) {
            hb[(size_t)b].c[a] = bubbles[b].center[a];
            hb[(size_t)b].lo[a] = bubbles[b].box_lo[a];
            hb[(size_t)b].hi[a] = bubbles[b].box_hi[a];
        }
        hb[(size_t)b].radius = bubbles[b].radius;
    }
    CloudIC ic;
    ic.thickness = p->thickness;
    ic.sharpness = p->sharpness;
    ic.zero_below = p->zero_below;
    ic.pulse_width = p->pulse_width;
    ic.rho_liquid = p->rho_liquid;
    ic.rho_gas = p->rho_gas;
    ic.p_ambient = p->p_ambient;
    ic.p_pulse = p->p_pulse;
    ic.nbubbles = nbubbles;
    BubbleIC* dev = nullptr;
    cudaError_t e = cudaMalloc(&dev, sizeof(BubbleIC) * hb.size());
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dev, hb.data(), sizeof(BubbleIC) * hb.size(), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
        const long long blocks = (s->ncell + 255) / 256;
        ic_bubble_cloud_kernel<<<(unsigned)blocks, 256, 0, s->stream>>>(s->buf[s->cur], s->g, s->M, ic, dev);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(dev);
    return e == cudaSuccess ? DIMGPU_OK : session_cuda_fail(s, e, "dimgpu_init_bubble_cloud");
}

}  // extern "C"
