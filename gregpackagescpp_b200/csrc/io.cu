// Host arrays <-> device bodies.
//
// The caller's arrays are the reference's layout (x3 / v3 / a3 as x, y, z triples per body, and one
// double per body for m, r, rest), in upload order.  The device keeps double4 records, possibly in a
// spatial order.  The conversion runs on the GPU: each requested array crosses PCIe once, as is,
// into (or out of) a device staging area, and a kernel packs (or unpacks and reorders) it, so the
// host does no per-body work.
#include <cuda_runtime.h>

#include <vector>

#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kIT = 256;

// Staging layout (doubles): x3 [3n] | v3 [3n] | a3 [3n] | m [n] | r [n] | rest [n] | rows (int32) [n]
struct IoView {
    double *x3, *v3, *a3, *m, *r, *rest;
    int32_t *rows;
};

static IoView io_view(double *base, int64_t n) {
    IoView v;
    v.x3 = base;
    v.v3 = base + 3 * n;
    v.a3 = base + 6 * n;
    v.m = base + 9 * n;
    v.r = base + 10 * n;
    v.rest = base + 11 * n;
    v.rows = reinterpret_cast<int32_t *>(base + 12 * n);
    return v;
}

static int ensure_io(gtd_system *s, int64_t n) {
    const size_t need = sizeof(double) * (size_t)(12 * n + (n + 1) / 2 + 1);
    if (need <= s->io_bytes) return GTD_OK;
    cudaFree(s->io_dev);
    s->io_dev = nullptr;
    s->io_bytes = 0;
    GTD_CUDA(cudaMalloc(&s->io_dev, need));
    s->io_bytes = need;
    return GTD_OK;
}

// bad[0] / bad[1]: first body with a negative mass / radius (INT32_MAX when none).
__global__ void pack_bodies_kernel(int64_t n, const double *x3, const double *v3, const double *m, const double *r,
                                   const double *rest, int has_v, int has_r, int has_rest, double4 *pm, double4 *vel,
                                   double4 *acc, double *rad, double *rest_out, int32_t *ids, int *bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double mi = m[i];
    const double ri = has_r ? r[i] : 0.0;
    if (mi < 0) atomicMin(&bad[0], (int)i);
    if (ri < 0) atomicMin(&bad[1], (int)i);
    pm[i] = make_double4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], mi);
    vel[i] = has_v ? make_double4(v3[3 * i], v3[3 * i + 1], v3[3 * i + 2], 0.0) : make_double4(0.0, 0.0, 0.0, 0.0);
    acc[i] = make_double4(0.0, 0.0, 0.0, 0.0);
    rad[i] = ri;
    rest_out[i] = has_rest ? rest[i] : 1.0;
    ids[i] = (int32_t)i;
}

// Slot i goes to row rows[i] (or ids[i], or i) of each requested output.
__global__ void unpack_bodies_kernel(int64_t n, const double4 *pm, const double4 *vel, const double4 *acc,
                                     const double *rad, const double *rest, const int32_t *map, IoView o,
                                     unsigned want) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t w = map ? map[i] : i;
    if (want & 1) {
        const double4 p = pm[i];
        o.x3[3 * w] = p.x; o.x3[3 * w + 1] = p.y; o.x3[3 * w + 2] = p.z;
    }
    if (want & 2) {
        const double4 v = vel[i];
        o.v3[3 * w] = v.x; o.v3[3 * w + 1] = v.y; o.v3[3 * w + 2] = v.z;
    }
    if (want & 4) {
        const double4 a = acc[i];
        o.a3[3 * w] = a.x; o.a3[3 * w + 1] = a.y; o.a3[3 * w + 2] = a.z;
    }
    if (want & 8) o.m[w] = pm[i].w;
    if (want & 16) o.r[w] = rad[i];
    if (want & 32) o.rest[w] = rest[i];
}

// Slot i takes row rows[i] (or ids[i], or i) of each given input; acceleration and order untouched.
__global__ void update_bodies_kernel(int64_t n, double4 *pm, double4 *vel, double *rad, double *rest,
                                     const int32_t *map, IoView in, unsigned have) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t w = map ? map[i] : i;
    double4 p = pm[i];
    if (have & 1) { p.x = in.x3[3 * w]; p.y = in.x3[3 * w + 1]; p.z = in.x3[3 * w + 2]; }
    if (have & 8) p.w = in.m[w];
    pm[i] = p;
    if (have & 2) {
        double4 v = vel[i];
        v.x = in.v3[3 * w]; v.y = in.v3[3 * w + 1]; v.z = in.v3[3 * w + 2];
        vel[i] = v;
    }
    if (have & 16) rad[i] = in.r[w];
    if (have & 32) rest[i] = in.rest[w];
}

}  // namespace gtd

using namespace gtd;

void release_io(gtd_system *s) {
    cudaFree(s->io_dev);
    s->io_dev = nullptr;
    s->io_bytes = 0;
}

// Fills the device bodies from the caller's arrays (upload order); s->n etc. are set by the caller.
int device_upload(gtd_system *s, int64_t n, const double *m, const double *r, const double *rest, const double *x3,
                  const double *v3) {
    int rc = ensure_io(s, n);
    if (rc) return rc;
    IoView io = io_view(static_cast<double *>(s->io_dev), n);
    cudaStream_t st = s->stream;
    const size_t d = sizeof(double);
    GTD_CUDA(cudaMemcpyAsync(io.x3, x3, 3 * d * (size_t)n, cudaMemcpyHostToDevice, st));
    GTD_CUDA(cudaMemcpyAsync(io.m, m, d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (v3) GTD_CUDA(cudaMemcpyAsync(io.v3, v3, 3 * d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (r) GTD_CUDA(cudaMemcpyAsync(io.r, r, d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (rest) GTD_CUDA(cudaMemcpyAsync(io.rest, rest, d * (size_t)n, cudaMemcpyHostToDevice, st));
    int *bad = reinterpret_cast<int *>(io.rows);  // two ints of scratch, before the rows are needed
    const int init[2] = {INT32_MAX, INT32_MAX};
    GTD_CUDA(cudaMemcpyAsync(bad, init, sizeof init, cudaMemcpyHostToDevice, st));
    pack_bodies_kernel<<<(unsigned)((n + kIT - 1) / kIT), kIT, 0, st>>>(n, io.x3, io.v3, io.m, io.r, io.rest, v3 != nullptr,
                                                                      r != nullptr, rest != nullptr, s->pm[0], s->vel,
                                                                      s->acc, s->rad, s->rest, s->ids, bad);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    int hb[2] = {0, 0};
    GTD_CUDA(cudaMemcpyAsync(hb, bad, sizeof hb, cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaStreamSynchronize(st));
    if (hb[0] != INT32_MAX && hb[0] <= hb[1])
        return fail(GTD_ERR_INVALID_ARGUMENT, "negative mass at body %lld", (long long)hb[0]);
    if (hb[1] != INT32_MAX) return fail(GTD_ERR_INVALID_ARGUMENT, "negative radius at body %lld", (long long)hb[1]);
    return GTD_OK;
}

// Device slot -> host row map for the live bodies (NULL: identity), staged in io.rows when needed.
static int row_map(gtd_system *s, const IoView &io, const int32_t **map) {
    *map = nullptr;
    if (s->n != s->n_uploaded) {  // after merges: ranks of the surviving upload indices (host sort)
        std::vector<int64_t> row;
        int rc = output_rows(s, row);
        if (rc) return rc;
        std::vector<int32_t> r32(row.begin(), row.end());
        GTD_CUDA(cudaMemcpyAsync(io.rows, r32.data(), sizeof(int32_t) * (size_t)s->n, cudaMemcpyHostToDevice,
                                 s->stream));
        GTD_CUDA(cudaStreamSynchronize(s->stream));
        *map = io.rows;
    } else if (s->ordered) {
        *map = s->ids;
    }
    return GTD_OK;
}

// Writes the requested arrays (any may be NULL) in download order: upload order among the live bodies.
int device_download(gtd_system *s, double *m, double *r, double *rest, double *x3, double *v3, double *a3) {
    const int64_t n = s->n;
    int rc = ensure_io(s, n);
    if (rc) return rc;
    IoView io = io_view(static_cast<double *>(s->io_dev), n);
    cudaStream_t st = s->stream;
    const int32_t *map = nullptr;
    rc = row_map(s, io, &map);
    if (rc) return rc;
    const unsigned want = (x3 ? 1u : 0u) | (v3 ? 2u : 0u) | (a3 ? 4u : 0u) | (m ? 8u : 0u) | (r ? 16u : 0u) |
                          (rest ? 32u : 0u);
    if (!want) return GTD_OK;
    unpack_bodies_kernel<<<(unsigned)((n + kIT - 1) / kIT), kIT, 0, st>>>(n, s->pm[s->cur], s->vel, s->acc, s->rad,
                                                                        s->rest, map, io, want);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    const size_t d = sizeof(double);
    if (x3) GTD_CUDA(cudaMemcpyAsync(x3, io.x3, 3 * d * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (v3) GTD_CUDA(cudaMemcpyAsync(v3, io.v3, 3 * d * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (a3) GTD_CUDA(cudaMemcpyAsync(a3, io.a3, 3 * d * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (m) GTD_CUDA(cudaMemcpyAsync(m, io.m, d * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (r) GTD_CUDA(cudaMemcpyAsync(r, io.r, d * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (rest) GTD_CUDA(cudaMemcpyAsync(rest, io.rest, d * (size_t)n, cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaStreamSynchronize(st));
    return GTD_OK;
}

// Overwrites the given arrays (any may be NULL) of the live bodies, in download order, leaving the
// accelerations, the body order and the evolve state as they are.
int device_update(gtd_system *s, const double *m, const double *r, const double *rest, const double *x3,
                  const double *v3) {
    const int64_t n = s->n;
    const unsigned have = (x3 ? 1u : 0u) | (v3 ? 2u : 0u) | (m ? 8u : 0u) | (r ? 16u : 0u) | (rest ? 32u : 0u);
    if (n == 0 || !have) return GTD_OK;
    int rc = ensure_io(s, n);
    if (rc) return rc;
    IoView io = io_view(static_cast<double *>(s->io_dev), n);
    cudaStream_t st = s->stream;
    const int32_t *map = nullptr;
    rc = row_map(s, io, &map);
    if (rc) return rc;
    const size_t d = sizeof(double);
    if (x3) GTD_CUDA(cudaMemcpyAsync(io.x3, x3, 3 * d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (v3) GTD_CUDA(cudaMemcpyAsync(io.v3, v3, 3 * d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (m) GTD_CUDA(cudaMemcpyAsync(io.m, m, d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (r) GTD_CUDA(cudaMemcpyAsync(io.r, r, d * (size_t)n, cudaMemcpyHostToDevice, st));
    if (rest) GTD_CUDA(cudaMemcpyAsync(io.rest, rest, d * (size_t)n, cudaMemcpyHostToDevice, st));
    update_bodies_kernel<<<(unsigned)((n + kIT - 1) / kIT), kIT, 0, st>>>(n, s->pm[s->cur], s->vel, s->rad, s->rest,
                                                                        map, io, have);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    GTD_CUDA(cudaStreamSynchronize(st));  // the caller's arrays may change as soon as this returns
    if (x3 || m) s->tree_valid = false;
    return GTD_OK;
}
