// .nsys snapshots of a gtd::system: the reference's only on-disk format.
//
//   write: system::to_nsys            gregsys.hpp:3214-3258
//   read:  system::load_from_nsys     gregsys.hpp:947-1400 (validation order and messages kept)
//   layout: nsys_header / nsys_chunk  gregsys.hpp:1444-1477
//
// The file is a 96-byte header followed by one chunk per body and zero padding to a 4-byte
// boundary.  A chunk is the C struct { char r_coeff[16]; M mass; R radius; T x, y, z, vx, vy, vz; }
// with natural alignment, so its size and field offsets follow from sizeof(M), sizeof(R) and
// sizeof(T).  Long doubles (the restitution coefficient, the header's time and time-step, and M/R/T
// when they are long double) are the x86-64 80-bit extended format in 16 bytes.
//
// On the device the bodies live as SoA doubles.  Writing packs the chunks on the GPU (one thread per
// body, staged through shared memory so the global writes are whole coalesced words) and moves them
// in one device-to-host copy; reading moves the file's chunk bytes in one host-to-device copy and
// unpacks them on the GPU, with the NaN/Inf scan of the reference done by the same threads.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <string>
#include <utility>
#include <vector>

#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kNsysHeader = 96;
constexpr int kPackThreads = 128;

struct NsysLayout {
    int ms, rs, ts;           // sizes of M, R, T (4, 8 or 16)
    int off_m, off_r, off_t;  // byte offsets in the chunk (the T fields are contiguous)
    int bytes;                // sizeof(nsys_chunk)
};

static int align_of(int size) { return size; }  // float 4, double 8, x86-64 long double 16

static NsysLayout nsys_layout(int ms, int rs, int ts) {
    auto up = [](int x, int a) { return (x + a - 1) / a * a; };
    NsysLayout L{ms, rs, ts, 0, 0, 0, 0};
    int off = 16;  // char r_coeff[16]
    L.off_m = up(off, align_of(ms));
    off = L.off_m + ms;
    L.off_r = up(off, align_of(rs));
    off = L.off_r + rs;
    L.off_t = up(off, align_of(ts));
    off = L.off_t + 6 * ts;
    int al = align_of(ms);
    if (align_of(rs) > al) al = align_of(rs);
    if (align_of(ts) > al) al = align_of(ts);
    L.bytes = up(off, al);
    return L;
}

// ---- binary64 <-> x87 80-bit extended (sign, 15-bit exponent biased by 16383, 64-bit significand
// with an explicit integer bit), written from the two formats' definitions ---------------------------
__host__ __device__ inline void f64_to_x87(double v, unsigned char *dst) {
    unsigned long long b;
    memcpy(&b, &v, 8);
    const unsigned sign = (unsigned)(b >> 63);
    const int e = (int)((b >> 52) & 0x7ff);
    const unsigned long long f = b & ((1ull << 52) - 1);
    unsigned long long mant = 0;
    unsigned exp = 0;
    if (e == 0x7ff) {  // Inf or NaN: all-ones exponent, integer bit set, fraction carried over
        exp = 0x7fff;
        mant = (1ull << 63) | (f << 11);
    } else if (e == 0) {
        if (f != 0) {  // subnormal binary64: normal in the wider exponent range
            int k = 0;
            while (!((f << k) & (1ull << 63))) ++k;
            mant = f << k;
            exp = (unsigned)(16383 - 1011 - k);
        }
    } else {
        mant = (1ull << 63) | (f << 11);
        exp = (unsigned)(e - 1023 + 16383);
    }
    const unsigned short se = (unsigned short)((sign << 15) | exp);
    memcpy(dst, &mant, 8);
    memcpy(dst + 8, &se, 2);
    memset(dst + 10, 0, 6);
}

// Round-to-nearest-even conversion of an x87 extended value to binary64.
__host__ __device__ inline double x87_to_f64(const unsigned char *src) {
    unsigned long long mant;
    unsigned short se;
    memcpy(&mant, src, 8);
    memcpy(&se, src + 8, 2);
    const unsigned long long sign = (unsigned long long)(se >> 15) << 63;
    const int X = se & 0x7fff;
    unsigned long long out;
    if (X == 0x7fff) {
        const unsigned long long frac = mant & ~(1ull << 63);
        out = frac == 0 ? (0x7ffull << 52) : ((0x7ffull << 52) | (1ull << 51) | (frac >> 11));
    } else if (mant == 0) {
        out = 0;
    } else {
        int k = 0;
        while (!((mant << k) & (1ull << 63))) ++k;
        const unsigned long long m = mant << k;
        int E = (X == 0 ? -16382 : X - 16383) - k;  // value = (m / 2^63) * 2^E
        if (E > 1023) {
            out = 0x7ffull << 52;
        } else if (E >= -1022) {
            unsigned long long q = m >> 11;  // 53 significant bits
            const unsigned long long rem = m & 0x7ff;
            if (rem > 0x400 || (rem == 0x400 && (q & 1))) ++q;
            if (q >> 53) {  // the rounding carried into a new leading bit
                q >>= 1;
                ++E;
            }
            out = E > 1023 ? (0x7ffull << 52) : ((unsigned long long)(E + 1023) << 52) | (q & ((1ull << 52) - 1));
        } else {
            const int sh = -(E + 1011);  // q = m * 2^(E + 1011), a subnormal significand
            if (sh >= 65) {
                out = 0;
            } else {
                unsigned long long q = sh >= 64 ? 0 : (m >> sh);
                const unsigned long long rem = sh >= 64 ? m : (m & ((1ull << sh) - 1));
                const unsigned long long half = 1ull << (sh - 1);
                if (rem > half || (rem == half && (q & 1))) ++q;
                out = q;  // q == 2^52 is the smallest normal, whose bits are the same
            }
        }
    }
    out |= sign;
    double d;
    memcpy(&d, &out, 8);
    return d;
}

__device__ inline void put_real(unsigned char *dst, double v, int size) {
    if (size == 4) {
        const float f = __double2float_rn(v);
        memcpy(dst, &f, 4);
    } else if (size == 8) {
        memcpy(dst, &v, 8);
    } else {
        f64_to_x87(v, dst);
    }
}

__device__ inline double get_real(const unsigned char *src, int size) {
    if (size == 4) {
        float f;
        memcpy(&f, src, 4);
        return (double)f;
    }
    if (size == 8) {
        double d;
        memcpy(&d, src, 8);
        return d;
    }
    return x87_to_f64(src);
}

// One thread per body: the chunk is assembled in shared memory, then the block's chunks leave as
// consecutive 4-byte words (every chunk size is a multiple of 4).
__global__ void __launch_bounds__(kPackThreads) nsys_pack_kernel(int64_t n, NsysLayout L, const double4 *pm,
                                                                 const double4 *vel, const double *rad,
                                                                 const double *rest, unsigned char *out) {
    extern __shared__ __align__(16) unsigned char stage[];
    const int64_t b0 = (int64_t)blockIdx.x * kPackThreads;
    const int cnt = (int)min((int64_t)kPackThreads, n - b0);
    const int t = threadIdx.x;
    if (t < cnt) {
        const int64_t i = b0 + t;
        unsigned char *c = stage + (size_t)t * L.bytes;
        for (int k = 0; k < L.bytes; ++k) c[k] = 0;
        f64_to_x87(rest[i], c);
        const double4 p = pm[i], v = vel[i];
        put_real(c + L.off_m, p.w, L.ms);
        put_real(c + L.off_r, rad[i], L.rs);
        const double f[6] = {p.x, p.y, p.z, v.x, v.y, v.z};
#pragma unroll
        for (int k = 0; k < 6; ++k) put_real(c + L.off_t + k * L.ts, f[k], L.ts);
    }
    __syncthreads();
    const int words = cnt * L.bytes / 4;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(stage);
    uint32_t *dst = reinterpret_cast<uint32_t *>(out + (size_t)b0 * L.bytes);
    for (int w = t; w < words; w += kPackThreads) dst[w] = src[w];
}

// The reverse, with the reference's NaN/Inf scan (gregsys.hpp:1309-1334): the first offending chunk
// and, within it, the first field in the order r_coeff, mass, radius, xpos ... zvel.
__global__ void __launch_bounds__(kPackThreads) nsys_unpack_kernel(int64_t n, NsysLayout L, int rest_size,
                                                                   int check, const unsigned char *in, double4 *pm,
                                                                   double4 *vel, double *rad, double *rest,
                                                                   int32_t *ids, unsigned long long *bad) {
    extern __shared__ __align__(16) unsigned char stage[];
    const int64_t b0 = (int64_t)blockIdx.x * kPackThreads;
    const int cnt = (int)min((int64_t)kPackThreads, n - b0);
    const int t = threadIdx.x;
    const int words = cnt * L.bytes / 4;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(in + (size_t)b0 * L.bytes);
    uint32_t *dst = reinterpret_cast<uint32_t *>(stage);
    for (int w = t; w < words; w += kPackThreads) dst[w] = src[w];
    __syncthreads();
    if (t >= cnt) return;
    const int64_t i = b0 + t;
    const unsigned char *c = stage + (size_t)t * L.bytes;
    double f[9];
    f[0] = get_real(c, rest_size);
    f[1] = get_real(c + L.off_m, L.ms);
    f[2] = get_real(c + L.off_r, L.rs);
#pragma unroll
    for (int k = 0; k < 6; ++k) f[3 + k] = get_real(c + L.off_t + k * L.ts, L.ts);
    if (check) {
        for (int k = 0; k < 9; ++k) {
            if (!isfinite(f[k])) {
                atomicMin(bad, ((unsigned long long)i << 4) | (unsigned long long)k);
                break;
            }
        }
    }
    pm[i] = make_double4(f[3], f[4], f[5], f[1]);
    vel[i] = make_double4(f[6], f[7], f[8], 0.0);
    rad[i] = f[2];
    rest[i] = f[0];
    ids[i] = (int32_t)i;
}

static int ensure_nsys_buffers(gtd_system *s, size_t bytes) {
    if (bytes > s->nsys_dev_bytes) {
        cudaFree(s->nsys_dev);
        s->nsys_dev = nullptr;
        s->nsys_dev_bytes = 0;
        GTD_CUDA(cudaMalloc(&s->nsys_dev, bytes));
        s->nsys_dev_bytes = bytes;
    }
    if (bytes > s->nsys_host_bytes) {
        cudaFreeHost(s->nsys_host);
        s->nsys_host = nullptr;
        s->nsys_host_bytes = 0;
        GTD_CUDA(cudaMallocHost(&s->nsys_host, bytes));
        s->nsys_host_bytes = bytes;
    }
    return GTD_OK;
}

static bool valid_size(int z) { return z == 4 || z == 8 || z == 16; }

static uint64_t nsys_file_size(uint64_t n, int chunk_bytes) {  // gregsys.hpp:943-946
    const uint64_t body = n * (uint64_t)chunk_bytes;
    const int rem = (int)(body % 4);
    return kNsysHeader + body + (rem ? 4 - rem : 0);
}

// Enqueues the packing of the live bodies (in output order) and its copy into pinned buffer w,
// then the event that marks the copy done.  Nothing waits here.
static int pack_async(gtd_system *s, const NsysLayout &L, gtd_system::NsysWrite &w) {
    const int64_t n = s->n;
    int rc = restore_upload_order(s);  // output row order
    if (rc) return rc;
    const size_t bytes = (size_t)n * L.bytes;
    if (bytes > s->nsys_dev_bytes) {
        cudaFree(s->nsys_dev);
        s->nsys_dev = nullptr;
        s->nsys_dev_bytes = 0;
        GTD_CUDA(cudaMalloc(&s->nsys_dev, bytes));
        s->nsys_dev_bytes = bytes;
    }
    if (bytes > w.bytes) {
        cudaFreeHost(w.buf);
        w.buf = nullptr;
        w.bytes = 0;
        GTD_CUDA(cudaMallocHost(&w.buf, bytes));
        w.bytes = bytes;
    }
    if (!w.done) GTD_CUDA(cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming));
    const unsigned blocks = (unsigned)((n + kPackThreads - 1) / kPackThreads);
    nsys_pack_kernel<<<blocks, kPackThreads, (size_t)kPackThreads * L.bytes, s->stream>>>(
        n, L, s->pm[s->cur], s->vel, s->rad, s->rest, static_cast<unsigned char *>(s->nsys_dev));
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    GTD_CUDA(cudaMemcpyAsync(w.buf, s->nsys_dev, bytes, cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaEventRecord(w.done, s->stream));
    return GTD_OK;
}

// The host side of one write: the header, the chunks once their copy is done, the padding.
static std::pair<int, std::string> write_file(int device, cudaEvent_t done, std::string path,
                                              std::vector<unsigned char> header, const void *body, size_t body_bytes,
                                              int64_t *written) {
    *written = 0;
    if (body_bytes) {
        cudaSetDevice(device);
        const cudaError_t e = cudaEventSynchronize(done);
        if (e != cudaSuccess) return {GTD_ERR_CUDA, std::string("snapshot copy: ") + cudaGetErrorString(e)};
    }
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return {GTD_OK, ""};  // the reference returns 0 when the stream does not open
    bool ok = std::fwrite(header.data(), 1, header.size(), f) == header.size();
    int64_t tell = (int64_t)header.size();
    if (ok && body_bytes) {
        ok = std::fwrite(body, 1, body_bytes, f) == body_bytes;
        tell += (int64_t)body_bytes;
        if (const int rem = (int)(tell % 4); ok && rem) {
            static const unsigned char zeros[4] = {0, 0, 0, 0};
            ok = std::fwrite(zeros, 1, (size_t)(4 - rem), f) == (size_t)(4 - rem);
            tell += 4 - rem;
        }
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) return {GTD_ERR_INVALID_ARGUMENT, "error writing " + path};
    *written = tell;
    return {GTD_OK, ""};
}

// Waits for the write in slot k (if any); its status, with the message set for the caller's thread.
static int finish_write(gtd_system *s, int k) {
    gtd_system::NsysWrite &w = s->nsys_w[k];
    if (!w.job.valid()) return GTD_OK;
    const std::pair<int, std::string> r = w.job.get();
    if (r.first) return fail(r.first, "%s", r.second.c_str());
    return GTD_OK;
}

}  // namespace gtd

using namespace gtd;

void release_nsys(gtd_system *s) {
    for (auto &w : s->nsys_w) {
        if (w.job.valid()) w.job.wait();
        cudaFreeHost(w.buf);
        if (w.done) cudaEventDestroy(w.done);
        w.buf = nullptr;
        w.bytes = 0;
        w.done = nullptr;
    }
    cudaFree(s->nsys_dev);
    cudaFreeHost(s->nsys_host);
    s->nsys_dev = nullptr;
    s->nsys_host = nullptr;
    s->nsys_dev_bytes = s->nsys_host_bytes = 0;
}

extern "C" {

int gtd_nsys_chunk_size(int m_size, int r_size, int t_size, int *chunk_bytes) {
    if (!chunk_bytes) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!valid_size(m_size) || !valid_size(r_size) || !valid_size(t_size))
        return fail(GTD_ERR_UNSUPPORTED, "M, R and T must be float, double or long double (sizes 4, 8, 16)");
    *chunk_bytes = nsys_layout(m_size, r_size, t_size).bytes;
    return GTD_OK;
}

int gtd_system_to_nsys_async(gtd_system *s, const char *path, double time_elapsed, double dt, const uint64_t *g_vals,
                             int m_size, int r_size, int t_size) {
    if (!s || !g_vals) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!valid_size(m_size) || !valid_size(r_size) || !valid_size(t_size))
        return fail(GTD_ERR_UNSUPPORTED, "M, R and T must be float, double or long double (sizes 4, 8, 16)");
    if (!path) return GTD_OK;  // gregsys.hpp:3220-3221
    DeviceGuard g(s->device);
    const int k = s->nsys_next;
    int rc = finish_write(s, k);  // the slot's previous write must release its buffer first
    if (rc) return rc;
    gtd_system::NsysWrite &w = s->nsys_w[k];
    const NsysLayout L = nsys_layout(m_size, r_size, t_size);
    const int64_t n = s->n;
    if (n > 0) {
        rc = pack_async(s, L, w);
        if (rc) return rc;
    }
    std::vector<unsigned char> h(kNsysHeader, 0);
    h[0] = 'N';
    h[1] = 'S';
    h[2] = (unsigned char)(1 + (1 << 1) + (1 << 2) + (1 << 3));  // floating time, M, R and T
    h[3] = 16;                                                  // sizeof(long double)
    f64_to_x87(time_elapsed, h.data() + 4);
    f64_to_x87(dt, h.data() + 20);
    h[36] = (unsigned char)m_size;
    h[37] = (unsigned char)r_size;
    h[38] = (unsigned char)t_size;
    h[39] = 16;
    std::memcpy(h.data() + 40, g_vals, 6 * sizeof(uint64_t));
    const uint64_t nb = (uint64_t)n;
    std::memcpy(h.data() + 88, &nb, 8);
    const size_t body = (size_t)n * L.bytes;
    w.job = std::async(std::launch::async, write_file, s->device, w.done, std::string(path), std::move(h), w.buf, body,
                       &w.written);
    s->nsys_last = k;
    s->nsys_next = k ^ 1;
    return GTD_OK;
}

int gtd_system_nsys_wait(gtd_system *s, int64_t *bytes_written) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (bytes_written) *bytes_written = 0;
    const int last = s->nsys_last;
    const int first = last < 0 ? 0 : last ^ 1;  // the older write first
    int rc = finish_write(s, first);
    const int rc2 = finish_write(s, first ^ 1);
    if (!rc) rc = rc2;
    if (rc) return rc;
    if (bytes_written && last >= 0) *bytes_written = s->nsys_w[last].written;
    return GTD_OK;
}

int gtd_system_to_nsys(gtd_system *s, const char *path, double time_elapsed, double dt, const uint64_t *g_vals,
                       int m_size, int r_size, int t_size, int64_t *bytes_written) {
    if (bytes_written) *bytes_written = 0;
    const int rc = gtd_system_to_nsys_async(s, path, time_elapsed, dt, g_vals, m_size, r_size, t_size);
    if (rc || !path) return rc;  // a NULL path writes nothing, as in the reference
    return gtd_system_nsys_wait(s, bytes_written);
}

int gtd_system_load_nsys(gtd_system *s, const char *path, int check_nan_inf, int m_size, int r_size, int t_size,
                         double *time_elapsed, double *dt, uint64_t *g_vals, double *G) {
    if (!s || !path) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!valid_size(m_size) || !valid_size(r_size) || !valid_size(t_size))
        return fail(GTD_ERR_UNSUPPORTED, "M, R and T must be float, double or long double (sizes 4, 8, 16)");
    struct stat st {};
    if (stat(path, &st) == -1) return fail(GTD_ERR_NSYS_LOAD, "Error obtaining .nsys file information. No data loaded.\n");
    if (!S_ISREG(st.st_mode))
        return fail(GTD_ERR_NSYS_LOAD, ".nsys file provided is not a regular file. Could not load data.\n");
    if (st.st_size < (off_t)kNsysHeader) return fail(GTD_ERR_NSYS_LOAD, "Insufficient .nsys file size. No data loaded.\n");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(GTD_ERR_NSYS_LOAD, "Error opening .nsys file. Could not load data.\n");
    struct Closer {
        FILE *f;
        ~Closer() { std::fclose(f); }
    } closer{f};
    unsigned char h[kNsysHeader];
    if (std::fread(h, 1, sizeof h, f) != sizeof h)
        return fail(GTD_ERR_NSYS_LOAD, "Insufficient .nsys file size. No data loaded.\n");
    if (h[0] != 'N' && h[1] != 'S')  // both must differ, as in gregsys.hpp:987
        return fail(GTD_ERR_NSYS_FORMAT, "Invalid .nsys format: invalid file signature.\n");
    const unsigned d_types = h[2];
    if (d_types & 0x40)
        return fail(GTD_ERR_NSYS_FORMAT, "Invalid .nsys format: msb occupied in d_types field (should be zero).\n");
    // NSYS_TYPE_CHECK for floating-point M, R, T (gregsys.hpp:997-1044)
    const struct {
        unsigned bit;
        const char *str, *type;
        int size, file_size;
    } checks[3] = {{0x02, "mass", "M", m_size, h[36]},
                   {0x04, "radius", "R", r_size, h[37]},
                   {0x08, "position and velocity", "T", t_size, h[38]}};
    for (const auto &c : checks) {
        if (!(d_types & c.bit))
            return fail(GTD_ERR_NSYS_LOAD,
                        "Invalid .nsys format: d_types field states that %s values are stored in floating-point "
                        "format, but template parameter %s is integral.\n",
                        c.str, c.type);
        if (c.file_size != c.size) {
            char msg[128];
            std::snprintf(msg, sizeof msg,
                          "Size mismatch error: size of %s template parameter (%d bytes) does not match its reported "
                          "size (%d bytes) in the .nsys file.\n",
                          c.type, c.size, c.file_size);
            return fail(GTD_ERR_NSYS_LOAD, "%s", msg);
        }
    }
    const int rest_size = h[39];
    if (rest_size > 16) {
        char msg[156];
        std::snprintf(msg, sizeof msg,
                      "Size mismatch error: coefficient of restitution data size (%d bytes) larger than widest "
                      "floating point data type available (long double = %d bytes).\n",
                      rest_size, 16);
        return fail(GTD_ERR_NSYS_FORMAT, "%s", msg);
    }
    if (rest_size != 16 && rest_size != 8 && rest_size != 4) {
        char msg[192];
        std::snprintf(msg, sizeof msg,
                      "Size mismatch error: coefficient of restitution data size (%d bytes) does not match any "
                      "floating point data type available:\nfloat = 4 bytes,\ndouble = 8 bytes,\nlong double = 16 "
                      "bytes.\n",
                      rest_size);
        return fail(GTD_ERR_NSYS_FORMAT, "%s", msg);
    }
    const NsysLayout L = nsys_layout(m_size, r_size, t_size);
    uint64_t n_file;
    std::memcpy(&n_file, h + 88, 8);
    if ((uint64_t)st.st_size != nsys_file_size(n_file, L.bytes)) {
        char msg[156];
        std::snprintf(msg, sizeof msg,
                      "Error: file size does not match expected file size based on number of bodies.\nExpected: %llu "
                      "bytes. Instead got: %zu bytes. No data loaded.\n",
                      (unsigned long long)nsys_file_size(n_file, L.bytes), (size_t)st.st_size);
        return fail(GTD_ERR_NSYS_FORMAT, "%s", msg);
    }
    // time point and time-step (gregsys.hpp:1111-1272)
    const int time_size = h[3];
    double t_el = 0.0, t_dt = 0.0;
    if (d_types & 0x01) {
        if (time_size == 16) {
            t_el = x87_to_f64(h + 4);
            t_dt = x87_to_f64(h + 20);
        } else if (time_size == 8) {
            std::memcpy(&t_el, h + 4, 8);
            std::memcpy(&t_dt, h + 20, 8);
        } else if (time_size == 4) {
            float a, b;
            std::memcpy(&a, h + 4, 4);
            std::memcpy(&b, h + 20, 4);
            t_el = a;
            t_dt = b;
        } else {
            char msg[212];
            std::snprintf(msg, sizeof msg,
                          "Size mismatch error: reported size of data type for time values in .nsys file (%d bytes) "
                          "does not match any floating point data type available:\nfloat = 4 bytes,\ndouble = 8 "
                          "bytes,\nlong double = 16 bytes.\n",
                          time_size);
            return fail(GTD_ERR_NSYS_FORMAT, "%s", msg);
        }
    } else {
        if (time_size > 8) {
            char msg[204];
            std::snprintf(msg, sizeof msg,
                          "Size mismatch error: reported size of data type for time values in .nsys file (%d bytes) "
                          "larger than largest unsigned integral data types available:\nuint64_t = 8 bytes,\n"
                          "unsigned long long = 8 bytes\n",
                          time_size);
            return fail(GTD_ERR_NSYS_FORMAT, "%s", msg);
        }
        unsigned long long a = 0, b = 0;
        std::memcpy(&a, h + 4, (size_t)time_size);
        std::memcpy(&b, h + 20, (size_t)time_size);
        t_el = (double)a;
        t_dt = (double)b;
    }
    if (check_nan_inf && !std::isfinite(t_dt)) return fail(GTD_ERR_NSYS_FORMAT, "Error: time-step is NaN or INF.");
    if (!(t_dt > 0)) return fail(GTD_ERR_INVALID_ARGUMENT, "Time-step cannot be zero or negative.\n");
    // G from the stored units (gregsys.hpp:1281-1284): 64-bit integer products, long double quotient
    uint64_t gv[6];
    std::memcpy(gv, h + 40, sizeof gv);
    long double Gl = 66743;
    Gl *= gv[0] * gv[2] * gv[2] * gv[2] * gv[4] * gv[4];
    Gl /= gv[1] * gv[3] * gv[3] * gv[3] * gv[5] * gv[5];
    Gl /= 1000000000000000ull;
    // bodies
    if (n_file > (uint64_t)INT32_MAX)
        return fail(GTD_ERR_CAPACITY, "body count %llu not supported", (unsigned long long)n_file);
    const int64_t n = (int64_t)n_file;
    DeviceGuard g(s->device);
    int rc = gtd_system_upload(s, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (rc) return rc;
    if (n > 0) {
        const size_t bytes = (size_t)n * L.bytes;
        rc = ensure_nsys_buffers(s, bytes);
        if (rc) return rc;
        if (std::fread(s->nsys_host, 1, bytes, f) != bytes)
            return fail(GTD_ERR_NSYS_LOAD, "Error reading .nsys file. Could not load data.\n");
        rc = ensure_body_capacity(s, n);
        if (rc) return rc;
        unsigned long long *bad = reinterpret_cast<unsigned long long *>(s->stage);  // pinned, >= 8 bytes
        GTD_CUDA(cudaMemcpyAsync(s->nsys_dev, s->nsys_host, bytes, cudaMemcpyHostToDevice, s->stream));
        unsigned long long *bad_dev = reinterpret_cast<unsigned long long *>(s->acc);  // scratch until zeroed
        GTD_CUDA(cudaMemsetAsync(bad_dev, 0xff, sizeof(unsigned long long), s->stream));
        const unsigned blocks = (unsigned)((n + kPackThreads - 1) / kPackThreads);
        nsys_unpack_kernel<<<blocks, kPackThreads, (size_t)kPackThreads * L.bytes, s->stream>>>(
            n, L, rest_size, check_nan_inf ? 1 : 0, static_cast<const unsigned char *>(s->nsys_dev), s->pm[0],
            s->vel, s->rad, s->rest, s->ids, bad_dev);
        GTD_CHECK_LAUNCH();
        s->launches += 1;
        GTD_CUDA(cudaMemcpyAsync(bad, bad_dev, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->stream));
        GTD_CUDA(cudaMemsetAsync(s->acc, 0, sizeof(double4) * (size_t)n, s->stream));
        GTD_CUDA(cudaStreamSynchronize(s->stream));
        if (*bad != ~0ull) {
            static const char *names[9] = {"r_coeff", "mass", "radius", "xpos", "ypos", "zpos", "xvel", "yvel", "zvel"};
            const unsigned long long idx = *bad >> 4;
            char msg[128];
            std::snprintf(msg, sizeof msg,
                          "Error: NaN or INF encountered in chunk with index %llu. Invalid field: \"%s\"\n", idx,
                          names[*bad & 15]);
            gtd_system_upload(s, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
            return fail(GTD_ERR_NSYS_LOAD, "%s", msg);
        }
        rc = set_loaded_bodies(s, n);
        if (rc) return rc;
    }
    if (time_elapsed) *time_elapsed = t_el;
    if (dt) *dt = t_dt;
    if (g_vals) std::memcpy(g_vals, gv, sizeof gv);
    if (G) *G = (double)Gl;
    return GTD_OK;
}

}  // extern "C"
