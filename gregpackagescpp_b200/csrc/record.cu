// Trajectory frames for systems with memFreq != 0.
//
// The reference keeps, per body, vectors of positions, velocities and kinetic energies
// (gregbod.hpp:304-320) and, per system, per-body potential and total energies and the system
// totals (gregsys.hpp:219-227), filled at every memFreq-th step by the integrators, the collision
// pass and calc_acc_and_e / calc_energy (gregsys.hpp:343-363, 439-476, 608-630).  Which of those
// records the reference actually makes depends on the method and on the collision mode; the host
// layers (include/gtd/gregsys.hpp, system.py) apply those rules.  The engine supplies the raw
// material: at every state s = 0, f, 2f, ... (<= the step count) of a direct-summation evolve it
// records one frame, holding for every body (in download order) x, y, z, vx, vy, vz,
// ke = 0.5 m |v| |v| (body::set_ke, gregbod.hpp:325-328) and pe = 0.5 sum_{j != i} -G m_i m_j / r_ij
// (cumulative_pe and the halving of gregsys.hpp:358-363, 464).  Each frame costs one O(N^2) FP64
// pass; it is copied to the host as soon as it is made.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kRT = 256;

// One thread per slot; the frame row is the body's upload index (no merges while recording).
__global__ void __launch_bounds__(kRT) frame_kernel(int64_t n, const double4 *pm, const double4 *vel,
                                                    const int32_t *ids, double G, double *out) {
    __shared__ double4 tile[kRT];
    const int t = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * kRT + t;
    double4 p = make_double4(0.0, 0.0, 0.0, 0.0), v = p;
    if (i < n) {
        p = pm[i];
        v = vel[i];
    }
    const double gm = G * p.w;
    double pe = 0.0;
    for (int64_t j0 = 0; j0 < n; j0 += kRT) {
        const int64_t j = j0 + t;
        tile[t] = j < n ? pm[j] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        const int lim = (int)min((int64_t)kRT, n - j0);
        for (int jj = 0; jj < lim; ++jj) {
            if (j0 + jj == i) continue;
            const double4 q = tile[jj];
            const double dx = __dsub_rn(q.x, p.x), dy = __dsub_rn(q.y, p.y), dz = __dsub_rn(q.z, p.z);
            const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
            pe = __dadd_rn(pe, -__ddiv_rn(__dmul_rn(gm, q.w), r));
        }
        __syncthreads();
    }
    if (i >= n) return;
    const double mag = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y)), __dmul_rn(v.z, v.z)));
    double *o = out + (size_t)ids[i] * 8;
    o[0] = p.x;
    o[1] = p.y;
    o[2] = p.z;
    o[3] = v.x;
    o[4] = v.y;
    o[5] = v.z;
    o[6] = __dmul_rn(__dmul_rn(__dmul_rn(0.5, p.w), mag), mag);
    o[7] = __dmul_rn(pe, 0.5);
}

}  // namespace gtd

using namespace gtd;

void release_record(gtd_system *s) {
    cudaFree(s->rec_dev);
    s->rec_dev = nullptr;
    s->rec_dev_n = 0;
    s->rec_frames.clear();
    s->rec_frames.shrink_to_fit();
    s->rec_states.clear();
}

// Appends the frame of the current (synchronised) state, labelled with its step index.
int record_frame(gtd_system *s, uint64_t state) {
    const int64_t n = s->n;
    if (n == 0) return GTD_OK;
    if (n != s->n_uploaded)
        return fail(GTD_ERR_UNSUPPORTED, "trajectory recording needs the uploaded bodies (none merged)");
    if (s->rec_dev_n < n) {
        cudaFree(s->rec_dev);
        s->rec_dev = nullptr;
        s->rec_dev_n = 0;
        GTD_CUDA(cudaMalloc(&s->rec_dev, sizeof(double) * 8 * (size_t)n));
        s->rec_dev_n = n;
    }
    const unsigned blocks = (unsigned)((n + kRT - 1) / kRT);
    frame_kernel<<<blocks, kRT, 0, s->stream>>>(n, s->pm[s->cur], s->vel, s->ids, s->G, s->rec_dev);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    // the pinned staging area holds 16 doubles per body
    GTD_CUDA(cudaMemcpyAsync(s->stage, s->rec_dev, sizeof(double) * 8 * (size_t)n, cudaMemcpyDeviceToHost,
                             s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    const double *h = reinterpret_cast<const double *>(s->stage);
    s->rec_frames.insert(s->rec_frames.end(), h, h + 8 * (size_t)n);
    s->rec_states.push_back((int64_t)state);
    s->rec_n = n;
    return GTD_OK;
}

extern "C" {

int gtd_system_set_recording(gtd_system *s, uint64_t every) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    s->rec_every = every;
    s->rec_frames.clear();
    s->rec_states.clear();
    return GTD_OK;
}

int gtd_system_recording(gtd_system *s, int64_t *frames, int64_t *n, int64_t *states, double *frame8) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    const int64_t f = (int64_t)s->rec_states.size();
    if (frames) *frames = f;
    if (n) *n = f ? s->rec_n : 0;
    if (states && f) std::memcpy(states, s->rec_states.data(), sizeof(int64_t) * (size_t)f);
    if (frame8 && f) std::memcpy(frame8, s->rec_frames.data(), sizeof(double) * s->rec_frames.size());
    return GTD_OK;
}

}  // extern "C"
