// C ABI of libzlfft_cuda (declared in include/zlfft.h).
//
// A plan owns, on its device: the unified twiddle table of its CFFT length
// (generated here in FP64 and rounded to the plan precision, G1), the RFFT
// split twiddles, and pinned host staging buffers for the
// host-pointer calls that mirror zldsp::fft::CFFT/RFFT member functions.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/zlfft.h"
#include "zlfft_istft.cuh"
#include "zlfft_launch.cuh"
#include "zlfft_macro.cuh"
#include "zlfft_mixed.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// A failed runtime call leaves its error pending for the next
// cudaGetLastError(), which would then report it against a later, successful
// launch; the failure paths below clear it once they have recorded it.
int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    return fail(ZLFFT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int alloc_fail(const char* what, size_t bytes) {
    cudaGetLastError();
    return fail(ZLFFT_ERR_ALLOC, "%s allocation of %zu bytes failed", what, bytes);
}

#define ZL_CUDA(call)                                  \
    do {                                               \
        cudaError_t _e = (call);                       \
        if (_e != cudaSuccess) return cuda_fail(_e, #call); \
    } while (0)

// ------------------------------------------------------------------ G1: twiddles
// Generated on the device in FP64 with the reference's own formula, then
// rounded to F: cospi(a) = cos(a * pi), sinpi(a) = sin(a * pi) with a*pi
// rounded to double first (src/common/zldsp_fft_common_math.hpp:19-24). This
// keeps the reference's values where a more accurate sincospi(a) would not:
// e.g. its cos(pi/2) entry is 6.1e-17, not 0. In FP32 the rounded table is
// bit-identical to the reference's, which makes the plain form's output
// bit-identical too.
__device__ __forceinline__ double ref_cospi(double a) { return cos(__dmul_rn(a, 3.141592653589793)); }
__device__ __forceinline__ double ref_sinpi(double a) { return sin(__dmul_rn(a, 3.141592653589793)); }

// T[t] = exp(-2*pi*i*t/M) for t < 3M/4, a = -2t/M
// (src/common/zldsp_fft_common_init.hpp:138-162: per stage the reference
// evaluates cospi(k * (-2/(4L)) * m), which is exactly a for t = m*k*M/(4L)).
template <typename F>
__global__ void twiddle_kernel(zlfft::Cx<F>* tw, int order, long long count) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const double a = (double)t * (-2.0 / (double)(1LL << order));
    zlfft::Cx<F> w;
    w.x = (F)ref_cospi(a);
    w.y = (F)ref_sinpi(a);
    tw[t] = w;
}

// RFFT split twiddles k = 0..M/2 for real length Nr = 2M, stored as pairs
// (wc, ws): wc = 0.5*cos(2 pi k / Nr), ws = 0.5*sin(2 pi k / Nr) + 0.5, FP64
// then rounded (src/common/zldsp_fft_common_init.hpp:374-381). Index 0 unused.
template <typename F>
__global__ void rfft_twiddle_kernel(zlfft::Cx<F>* rw, int rfft_order, long long count) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double a = (double)k * (2.0 / (double)(1LL << rfft_order));
    zlfft::Cx<F> w;
    w.x = (F)__dmul_rn(0.5, ref_cospi(a));
    w.y = (F)__dadd_rn(__dmul_rn(0.5, ref_sinpi(a)), 0.5);
    rw[k] = w;
}

// Per-stage tables (layout in zlfft_tile.cuh, stage_l0): entry r of the stage
// with sub-length L is W_{4L}^{q k} = T[q*k*M/(4L)] with q = r/L + 1, k = r%L,
// copied from the unified table T so the bits are identical.
template <typename F>
__global__ void stage_table_kernel(zlfft::Cx<F>* tws, const zlfft::Cx<F>* tw, int order, long long count) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const long long l0 = zlfft::stage_l0(order);
    long long L = l0;
    while (4 * L - l0 <= idx) L *= 4;  // stage containing idx: offset L - l0, size 3L
    const long long r = idx - (L - l0);
    const long long q = r / L + 1, k = r % L;
    const long long m = 1LL << order;
    tws[idx] = tw[q * k * (m / (4 * L))];
}

// Twiddles of one tensor-core pass with L_in > 1 (layout in zlfft_tc_pass.cuh),
// copied from the unified table so the values are the ones the kernel would
// otherwise read there.
__global__ void tc_pass_table_kernel(float2* out, const float2* T, int n, int l_in) {
    const int idx = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (idx < 4 * l_in) {
        const uint32_t k = (uint32_t)(idx >> 2), b = (uint32_t)(idx & 3);
        out[idx] = zlfft::tw_any(T, ((1u << b) * k) * (uint32_t)(n / (16 * l_in)), (uint32_t)n);
    } else if (idx < 20 * l_in) {
        const uint32_t r = (uint32_t)(idx - 4 * l_in), k = r >> 4, j = r & 15;
        out[idx] = zlfft::tw_any(T, (j * k) * (uint32_t)(n / (256 * l_in)), (uint32_t)n);
    }
}

// Self-test of the bounded-wait path: one CTA waits on an mbarrier that no
// one ever arrives at, with a short poll limit; the wait gives up, the kernel
// records kDevErrWaitTimeout in the error word and returns normally.
__global__ void selftest_wait_kernel(int* err, uint32_t limit) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        zlfft::mbar_init(&bar, 1);
        zlfft::fence_mbar_init();
    }
    __syncthreads();
    const bool ok = zlfft::mbar_wait(&bar, 0, limit);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(err, zlfft::kDevErrWaitTimeout);
}

}  // namespace
namespace zlfft {
cudaError_t tc_selftest_launch(const float2* in, float2* out, const float2* tw16, int* err, cudaStream_t st);
}
namespace {

struct TablesHolder {
    zlfft::TileTable f32{};
    zlfft::TileTable f64{};
    zlfft::PassTable p32{};
    zlfft::PassTable p64{};
    zlfft::PassTable p32s{};  // pass scheme 1, orders 19-20
    zlfft::PassTable p64s{};
    zlfft::GatherTable g32{};
    zlfft::GatherTable g64{};
    zlfft::TcPassTable tc{};
    zlfft::IstftTable i32{};
    zlfft::IstftTable i64{};
    zlfft::MacroTable m32{};
    zlfft::MacroTable m64{};
    TablesHolder() {
        zlfft::fill_macro_dif_f32(m32);
        zlfft::fill_macro_seg_f32(m32);
        zlfft::fill_macro_dif_f64(m64);
        zlfft::fill_macro_seg_f64(m64);
        zlfft::fill_istft_f32(i32);
        zlfft::fill_istft_f64(i64);
        zlfft::fill_tc_pass_a(tc);
        zlfft::fill_tc_pass_b(tc);
        zlfft::fill_tc_pass_c(tc);
        zlfft::fill_gather_f32(g32);
        zlfft::fill_gather_f64(g64);
        zlfft::fill_tile_c2c_f32(f32);
        zlfft::fill_tile_r2c_f32(f32);
        zlfft::fill_tile_c2c_f64(f64);
        zlfft::fill_tile_r2c_f64(f64);
        zlfft::fill_pass_f32_a(p32);
        zlfft::fill_pass_f32_b(p32);
        zlfft::fill_pass_f32_c(p32);
        zlfft::fill_pass_f64_a(p64);
        zlfft::fill_pass_f64_b(p64);
        zlfft::fill_pass_f64_c(p64);
        zlfft::fill_pass_split_f32(p32s);
        zlfft::fill_pass_split_f64(p64s);
    }
};

const TablesHolder& tables() {
    static TablesHolder t;
    return t;
}


// ------------------------------------------------------------------ autotuning table
// Process-wide: (device, kind, precision, order) -> the plan parameters that
// measured fastest there (zlfft_autotune), or that a tuning file recorded.
struct TuneEntry {
    int chunk_mb = 48, streams = 2, tma = 1, form = ZLFFT_MODE_PLAIN, split_fused = 0, store_tma = -1;
    double gbs = 0, gbs_default = 0;
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, TuneEntry> g_tune;
std::once_flag g_tune_env_once[64];

bool tune_lookup(int device, int kind, int prec, int order, TuneEntry* e) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(std::make_tuple(device, kind, prec, order));
    if (it == g_tune.end()) return false;
    *e = it->second;
    return true;
}

// GPU identity written into tuning files: name (spaces as '_') and SM count.
int gpu_identity(int device, std::string* name, int* sms) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    std::string n = prop.name;
    for (char& c : n)
        if (c == ' ' || c == '\t') c = '_';
    *name = n;
    *sms = prop.multiProcessorCount;
    return ZLFFT_OK;
}

int tuning_load_impl(int device, const char* path, size_t* loaded) {
    if (loaded) *loaded = 0;
    FILE* f = fopen(path, "r");
    if (!f) return fail(ZLFFT_ERR_INVALID_ARG, "cannot open tuning file %s", path);
    std::string name;
    int sms = 0;
    int rc = gpu_identity(device, &name, &sms);
    if (rc) {
        fclose(f);
        return rc;
    }
    char line[512];
    bool same_gpu = false;
    size_t n = 0;
    while (fgets(line, sizeof(line), f)) {
        char gname[256];
        int gsms = 0;
        if (sscanf(line, "gpu %255s sms %d", gname, &gsms) == 2) {
            same_gpu = (name == gname && sms == gsms);
            continue;
        }
        int kind, prec, order, chunk, streams, tma, form, fused, store;
        double gbs, gbs0;
        if (sscanf(line, "entry %d %d %d %d %d %d %d %d %d %lf %lf", &kind, &prec, &order, &chunk, &streams, &tma,
                   &form, &fused, &store, &gbs, &gbs0) != 11)
            continue;
        if (!same_gpu) continue;
        const bool ok = (kind == ZLFFT_C2C || kind == ZLFFT_R2C) && (prec == ZLFFT_F32 || prec == ZLFFT_F64) &&
                        order >= 0 && order <= zlfft::kPassMaxP + 1 && chunk >= 0 && chunk <= 4096 &&
                        (streams == 1 || streams == 2) && (tma == 0 || tma == 1) && (fused == 0 || fused == 1) &&
                        (store >= -1 && store <= 1) &&
                        (form == ZLFFT_MODE_PLAIN || form == ZLFFT_MODE_FAST ||
                         (form == ZLFFT_MODE_TC_FP16 && kind == ZLFFT_C2C && prec == ZLFFT_F32));
        if (!ok) continue;
        TuneEntry e;
        e.chunk_mb = chunk;
        e.streams = streams;
        e.tma = tma;
        e.form = form;
        e.split_fused = fused;
        e.store_tma = store;
        e.gbs = gbs;
        e.gbs_default = gbs0;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[std::make_tuple(device, kind, prec, order)] = e;
        ++n;
    }
    fclose(f);
    if (loaded) *loaded = n;
    return ZLFFT_OK;
}
}  // namespace

struct zlfft_plan_s {
    int kind = 0;
    int prec = 0;
    int order = 0;       // transform order (RFFT: real length)
    int cfft_order = 0;  // inner complex FFT order
    int mode = 0;
    int device = 0;
    int num_sms = 0;
    size_t esize = 0;  // bytes of one real
    void* d_tw = nullptr;
    size_t tw_count = 0;
    void* d_tws = nullptr;  // per-stage twiddle tables
    void* d_rw = nullptr;   // RFFT split twiddle pairs
    void* d_tctw = nullptr;  // tensor-core pass twiddles (MODE_TC_FP16), one section per pass
    size_t tctw_off[zlfft::kMaxPasses] = {0, 0, 0};  // element offset of each pass's section
    // host staging
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;
    void* h_in = nullptr;
    void* h_out = nullptr;
    void* d_in = nullptr;
    void* d_out = nullptr;
    size_t stage_in_bytes = 0, stage_out_bytes = 0;
    cudaEvent_t ev_host = nullptr;  // orders the chunks' transforms across the two staging streams
    int* h_err = nullptr;           // page-locked copy of the device error word (host path)
    // single small transforms from host buffers: page-locked buffers mapped into the device's address
    // space, read and written by the kernel directly (exec_host_small)
    void* hm_in = nullptr;
    void* hm_out = nullptr;
    int* hm_err = nullptr;  // the kernel's error word for those calls, mapped too
    size_t hm_in_bytes = 0, hm_out_bytes = 0;
    void* dm_in = nullptr;   // their device addresses
    void* dm_out = nullptr;
    void* dm_err = nullptr;
    std::atomic<size_t> launches{0};
    // multi-pass scratch (two buffers of `chunk` transforms each)
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaStream_t lanes[2] = {nullptr, nullptr};  // chunk pipelines (alternate chunks)
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    size_t chunk = 0;  // transforms per chunk; intermediates of one chunk stay L2-resident
    int* d_err = nullptr;  // device error word written by kernels (bounded waits that ran out)
    // plan parameters: defaults, or the device's tuning entry for this size
    size_t chunk_mb = 48;   // scratch per chunk-pipeline buffer (measured plateau: 32-128 MiB)
    int nlanes = 2;         // chunk pipelines
    int use_tma = 1;        // TMA staging of kernel inputs (else direct loads)
    bool tc_form = false;   // 256-point passes in the tensor-core split form
    bool fast_form = false; // multi-pass radix-16 groups with fast twiddles (ZLFFT_MODE_FAST)
    bool fuse_split = false;  // RFFT forward: split fused into the last pass (else its own kernel)
    int pass_scheme = 0;      // multi-pass stage grouping (zlfft_pass.cuh): 1 = two passes for orders 19-20
    int store_tma = -1;       // first pass output by TMA tensor stores (-1: the precision's default)
    // The reference's algorithm switch (src/common/zldsp_fft_common_init.hpp:305-339), where the plan
    // follows one: a CFFT order >= switch_order runs the macro path (zlfft_macro.cuh) with this micro
    // order; -1: the micro-only Stockham path
    int micro = -1;
    int max_l1 = -1, switch_order = -1;  // the switch the plan follows (-1: none)
    void* d_mtw = nullptr;                // macro path: unified twiddle table of the micro order
    void* d_mtws = nullptr;               // macro path: per-stage tables of the micro order
    std::mutex mu;            // the host path's staging buffers and streams
    std::mutex scratch_mu;    // first-use creation of the scratch, lanes and their events
};

namespace {

// The multi-pass kernels of a plan's precision and pass scheme.
const zlfft::PassTable& pass_table(const zlfft_plan_s* p) {
    if (p->pass_scheme == 1) return p->prec == ZLFFT_F32 ? tables().p32s : tables().p64s;
    return p->prec == ZLFFT_F32 ? tables().p32 : tables().p64;
}

// Pass scheme of a multi-pass plan: CFFT orders 19-20 may run in two passes
// (512 | 1024 and 1024 | 1024 points) rather than three. The tensor-core form
// keeps scheme 0 (its kernels are 256-point passes), and so does the RFFT
// (its forward split fuses into a last pass of 128-byte unit rows).
// Default, from same-box measurements (GB/s, three -> two passes): FP32
// order 19 plain 1860 -> 1961, fast 2130 -> 2545, so order 19 takes two. Order
// 20 stays at three: fast 2276 -> 2333 is within run-to-run spread, plain
// 1913 -> 1813 is slower, and its second 1024-point pass cannot drop the
// intermediate from L2 (32-byte unit rows), which raises DRAM traffic from
// 1.09x to 1.61x the algorithmic bytes. FP64 is slower at both orders (its
// 1024-point passes run one CTA per SM). ZLFFT_PASS_SCHEME=0 / 1 forces three
// / two passes wherever both exist.
int default_pass_scheme(const zlfft_plan_s* p) {
    static const int forced = [] {
        const char* e = getenv("ZLFFT_PASS_SCHEME");
        return e ? (e[0] == '0' ? 0 : 1) : -1;
    }();
    const bool ok = p->kind == ZLFFT_C2C && !p->tc_form && p->cfft_order >= zlfft::kPassSplitMinP &&
                    p->cfft_order <= zlfft::kPassSplitMaxP;
    if (!ok) return 0;
    if (forced >= 0) return forced;
    return (p->prec == ZLFFT_F32 && p->cfft_order == 19) ? 1 : 0;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (dev >= 0 && dev != prev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

void release(zlfft_plan p) {
    if (!p) return;
    DeviceGuard g(p->device);
    if (p->d_tw) cudaFree(p->d_tw);
    if (p->d_tws) cudaFree(p->d_tws);
    if (p->d_rw) cudaFree(p->d_rw);
    if (p->d_tctw) cudaFree(p->d_tctw);
    if (p->d_mtw) cudaFree(p->d_mtw);
    if (p->d_mtws) cudaFree(p->d_mtws);
    if (p->d_err) cudaFree(p->d_err);
    if (p->d_scratch) cudaFree(p->d_scratch);
    for (int i = 0; i < 2; ++i) {
        if (p->lanes[i]) cudaStreamDestroy(p->lanes[i]);
        if (p->ev_join[i]) cudaEventDestroy(p->ev_join[i]);
    }
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_host) cudaEventDestroy(p->ev_host);
    if (p->d_in) cudaFree(p->d_in);
    if (p->d_out) cudaFree(p->d_out);
    if (p->h_in) cudaFreeHost(p->h_in);
    if (p->h_out) cudaFreeHost(p->h_out);
    if (p->h_err) cudaFreeHost(p->h_err);
    if (p->hm_in) cudaFreeHost(p->hm_in);
    if (p->hm_out) cudaFreeHost(p->hm_out);
    if (p->hm_err) cudaFreeHost(p->hm_err);
    if (p->stream) cudaStreamDestroy(p->stream);
    if (p->stream2) cudaStreamDestroy(p->stream2);
    delete p;
}

// Elements (of the buffer's own type) that one transform reads or writes.
struct Extents {
    size_t in_elems, out_elems;   // count of complex or real elements
    bool in_complex, out_complex; // element type
};

Extents extents(const zlfft_plan_s* p, int op) {
    const size_t n = size_t{1} << p->order;
    if (p->kind == ZLFFT_C2C) return {n, n, true, true};
    const size_t nb = n / 2 + 1;
    if (op == ZLFFT_FORWARD) return {n, nb, false, true};
    if (op == ZLFFT_FORWARD_SQR_MAG) return {n, nb, false, false};
    return {nb, n, true, false};
}

int validate_op(const zlfft_plan_s* p, int op, int in_layout, int out_layout) {
    if (op < ZLFFT_FORWARD || op > ZLFFT_FORWARD_SQR_MAG) return fail(ZLFFT_ERR_INVALID_ARG, "invalid op %d", op);
    if (op == ZLFFT_FORWARD_SQR_MAG && p->kind != ZLFFT_R2C)
        return fail(ZLFFT_ERR_INVALID_ARG, "forward_sqr_mag is an RFFT operation");
    if ((in_layout != ZLFFT_AOS && in_layout != ZLFFT_SOA) || (out_layout != ZLFFT_AOS && out_layout != ZLFFT_SOA))
        return fail(ZLFFT_ERR_INVALID_ARG, "invalid layout");
    return ZLFFT_OK;
}

int device_op_code(const zlfft_plan_s* p, int op) {
    if (p->kind == ZLFFT_C2C) return op == ZLFFT_FORWARD ? zlfft::kC2CFwd : zlfft::kC2CBwd;
    if (op == ZLFFT_FORWARD) return zlfft::kR2CFwd;
    if (op == ZLFFT_FORWARD_SQR_MAG) return zlfft::kR2CSqrMag;
    return zlfft::kC2RBwd;
}

bool aligned(const void* ptr, size_t a) { return (reinterpret_cast<uintptr_t>(ptr) % a) == 0; }

// Aliasing of a batched call. Every kernel reads a transform's whole input
// before it writes that transform's output, and transforms are disjoint, so
// an output may share memory with an input when both start at the same
// address with the same byte stride (in-place CFFT; the padded in-place RFFT
// whose real stride is 2 * (N/2 + 1)): each transform then overwrites only
// its own input. Any other overlap, with more than one transform, lets one
// transform's output overwrite another's input before it is read.
int check_aliasing(const zlfft_plan_s* p, const Extents& ex, bool in_soa, bool out_soa, const void* in0,
                   const void* in1, const void* out0, const void* out1, size_t batch, size_t in_stride,
                   size_t out_stride) {
    if (batch <= 1) return ZLFFT_OK;
    struct Span {
        uintptr_t lo, hi;
        size_t step;  // bytes from one transform to the next
    };
    auto span = [&](const void* ptr, size_t unit, size_t elems, size_t stride) {
        const uintptr_t lo = reinterpret_cast<uintptr_t>(ptr);
        return Span{lo, lo + ((batch - 1) * stride + elems) * unit, stride * unit};
    };
    const size_t in_unit = ex.in_complex && !in_soa ? 2 * p->esize : p->esize;
    const size_t out_unit = ex.out_complex && !out_soa ? 2 * p->esize : p->esize;
    Span ins[2], outs[2];
    int ni = 0, no = 0;
    ins[ni++] = span(in0, in_unit, ex.in_elems, in_stride);
    if (in_soa) ins[ni++] = span(in1, in_unit, ex.in_elems, in_stride);
    outs[no++] = span(out0, out_unit, ex.out_elems, out_stride);
    if (out_soa) outs[no++] = span(out1, out_unit, ex.out_elems, out_stride);
    for (int i = 0; i < ni; ++i)
        for (int o = 0; o < no; ++o) {
            const Span& a = ins[i];
            const Span& b = outs[o];
            if (a.lo < b.hi && b.lo < a.hi && !(a.lo == b.lo && a.step == b.step))
                return fail(ZLFFT_ERR_INVALID_ARG,
                            "input and output overlap across transforms (in place needs the same start and byte stride)");
        }
    return ZLFFT_OK;
}

// Scratch for the multi-pass orders: two buffers of `chunk` transforms. The
// chunk is sized so that one chunk's intermediates (both buffers) stay in
// L2 between the passes; it is reused chunk after chunk.
int ensure_scratch(zlfft_plan_s* p) {
    std::lock_guard<std::mutex> lock(p->scratch_mu);
    if (p->d_scratch) return ZLFFT_OK;
    const size_t cx = 2 * p->esize;
    const size_t n = size_t{1} << p->cfft_order;
    const size_t per = n * cx;
    size_t budget = p->chunk_mb << 20;  // bytes of one scratch buffer
    if (const char* env = getenv("ZLFFT_CHUNK_MB")) {
        const long v = atol(env);
        if (v > 0) budget = (size_t)v << 20;
    }
    size_t chunk = budget / per;
    if (chunk == 0) chunk = 1;
    // the streams and events first: d_scratch is set last, so a failure
    // leaves the plan as it was and a later call tries again
    for (int i = 0; i < 2; ++i) {
        if ((!p->lanes[i] && cudaStreamCreateWithFlags(&p->lanes[i], cudaStreamNonBlocking) != cudaSuccess) ||
            (!p->ev_join[i] && cudaEventCreateWithFlags(&p->ev_join[i], cudaEventDisableTiming) != cudaSuccess)) {
            cudaGetLastError();
            return fail(ZLFFT_ERR_CUDA, "stream creation failed");
        }
    }
    if (!p->ev_fork && cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return fail(ZLFFT_ERR_CUDA, "event creation failed");
    }
    const size_t bytes = 4 * chunk * per;  // two buffers for each of the two chunk pipelines
    void* d = nullptr;
    if (cudaMalloc(&d, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(ZLFFT_ERR_ALLOC, "scratch allocation of %zu bytes failed", bytes);
    }
    p->scratch_bytes = bytes;
    p->chunk = chunk;
    p->d_scratch = d;
    return ZLFFT_OK;
}

// Grid of the RFFT split / pre-step kernels: x covers one transform's M/2 + 1
// bin pairs in blocks of 256; y strides over the batch, with about 16 blocks
// per SM in all.
dim3 pair_grid(const zlfft_plan_s* p, int M, long long batch) {
    const long long gx = (M / 2 + 1 + 255) / 256;
    long long gy = ((long long)p->num_sms * 16 + gx - 1) / gx;
    if (gy > batch) gy = batch;
    if (gy > 65535) gy = 65535;
    if (gy < 1) gy = 1;
    return dim3((unsigned)gx, (unsigned)gy, 1);
}

template <typename F>
cudaError_t launch_split(const zlfft_plan_s* p, int dop, int out_layout, const void* z, void* o0, void* o1,
                         long long batch, long long out_stride, cudaStream_t st, const zlfft::LaunchCtx& ctx,
                         void* const* go0 = nullptr, void* const* go1 = nullptr) {
    using C = zlfft::Cx<F>;
    const int M = 1 << p->cfft_order;
    const dim3 grid = pair_grid(p, M, batch);
    const C* zc = static_cast<const C*>(z);
    const C* rw = static_cast<const C*>(p->d_rw);
    if (dop == zlfft::kR2CSqrMag)
        zlfft::rfft_split_kernel<F, zlfft::kR2CSqrMag, zlfft::kAoS><<<grid, 256, 0, st>>>(zc, o0, o1, rw, M, batch, M, out_stride, go0, go1);
    else if (out_layout == ZLFFT_AOS)
        zlfft::rfft_split_kernel<F, zlfft::kR2CFwd, zlfft::kAoS><<<grid, 256, 0, st>>>(zc, o0, o1, rw, M, batch, M, out_stride, go0, go1);
    else
        zlfft::rfft_split_kernel<F, zlfft::kR2CFwd, zlfft::kSoA><<<grid, 256, 0, st>>>(zc, o0, o1, rw, M, batch, M, out_stride, go0, go1);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

template <typename F>
cudaError_t launch_pre(const zlfft_plan_s* p, int in_layout, const void* i0, const void* i1, void* z, long long batch,
                       long long in_stride, cudaStream_t st, const zlfft::LaunchCtx& ctx,
                       const void* const* gi0 = nullptr, const void* const* gi1 = nullptr) {
    using C = zlfft::Cx<F>;
    const int M = 1 << p->cfft_order;
    const dim3 grid = pair_grid(p, M, batch);
    const C* rw = static_cast<const C*>(p->d_rw);
    if (in_layout == ZLFFT_AOS)
        zlfft::rfft_pre_kernel<F, zlfft::kAoS><<<grid, 256, 0, st>>>(i0, i1, static_cast<C*>(z), rw, M, batch, in_stride, M, gi0, gi1);
    else
        zlfft::rfft_pre_kernel<F, zlfft::kSoA><<<grid, 256, 0, st>>>(i0, i1, static_cast<C*>(z), rw, M, batch, in_stride, M, gi0, gi1);
    if (ctx.launches) ++*ctx.launches;
    return cudaGetLastError();
}

// Intermediates between passes are dropped from L2 once read (pass_kernel,
// discard_in); ZLFFT_L2_DISCARD=0 keeps them (comparison).
bool l2_discard_enabled() {
    static const bool on = [] {
        const char* e = getenv("ZLFFT_L2_DISCARD");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Kernel of pass pi: the tensor-core split-precision pass where the plan asks
// for it and one exists (256-point passes, FP32 AoS), else the plain pass.
zlfft::PassLaunchFn pick_pass(const zlfft_plan_s* p, int pi, bool fwd, int li, int lo) {
    const int P = p->cfft_order;
    if (p->tc_form && li == ZLFFT_AOS && lo == ZLFFT_AOS) {
        // the serial kernel (tc_pass_kernel, three CTAs per SM); ZLFFT_TC_PIPE=1 selects the
        // warp-specialised pipelined one (tc_pipe_kernel), measured slower on B200: its phases
        // get 4 warps each where the serial kernel runs 24 warps per SM through every phase
        static const bool pipe = [] {
            const char* e = getenv("ZLFFT_TC_PIPE");
            return e && e[0] == '1';
        }();
        const auto& tt = tables().tc;
        zlfft::PassLaunchFn f = pipe ? tt.pipe[P - zlfft::kPassMinP][pi][fwd ? 1 : 0] : nullptr;
        if (!f) f = tt.fn[P - zlfft::kPassMinP][pi][fwd ? 1 : 0];
        if (f) return f;
    }
    const zlfft::PassTable& t = pass_table(p);
    if (p->fast_form && li == ZLFFT_AOS && lo == ZLFFT_AOS) {
        zlfft::PassLaunchFn f = t.fast[P - zlfft::kPassMinP][pi][fwd ? 1 : 0];
        if (f) return f;
    }
    return t.fn[P - zlfft::kPassMinP][pi][fwd ? 1 : 0][li][lo];
}

// Orders above the tile kernel: chunks of transforms through 2-3 Stockham
// passes (zlfft_pass.cuh); RFFT orders add the split (forward) or the
// pre-step (backward) as a separate elementwise kernel on the N/2-point
// spectrum, with the reference's arithmetic.
int exec_multipass(zlfft_plan_s* p, int dop, int in_layout, int out_layout, const zlfft::TileArgs& a,
                   cudaStream_t st, const zlfft::LaunchCtx& ctx) {
    const int P = p->cfft_order;
    if (P < zlfft::kPassMinP || P > zlfft::kPassMaxP)
        return fail(ZLFFT_ERR_UNSUPPORTED, "order %d is above the supported maximum", p->order);
    int rc = ensure_scratch(p);
    if (rc) return rc;
    const zlfft::PassTable& t = pass_table(p);
    const auto& row = t.fn[P - zlfft::kPassMinP];
    int np = 0;
    while (np < zlfft::kMaxPasses && row[np][1][0][0]) ++np;
    const size_t cx = 2 * p->esize;
    const long long n = 1LL << P;
    char* s0 = nullptr;
    char* s1 = nullptr;
    const bool fwd = (dop == zlfft::kC2CFwd || dop == zlfft::kR2CFwd || dop == zlfft::kR2CSqrMag);
    const bool r2c = (dop == zlfft::kR2CFwd || dop == zlfft::kR2CSqrMag);
    const bool c2r = (dop == zlfft::kC2RBwd);
    const int il = (r2c) ? ZLFFT_AOS : in_layout;   // R2C: real input read as complex pairs
    const int ol = (c2r) ? ZLFFT_AOS : out_layout;  // C2R: real output written as complex pairs
    const size_t in_elem = (in_layout == ZLFFT_SOA && !r2c) ? p->esize : cx;
    const size_t out_elem = (out_layout == ZLFFT_SOA && !c2r) ? p->esize : cx;
    // Chunks alternate between two internal streams forked from (and joined
    // back to) the caller's stream, so one chunk's passes overlap the other's
    // launch gaps and wave tails. Each stream owns two scratch buffers.
    const long long nchunks = (a.batch + (long long)p->chunk - 1) / (long long)p->chunk;
    const bool fork = nchunks > 1 && p->nlanes > 1;
    if (fork) {
        if (cudaEventRecord(p->ev_fork, st) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "event record failed");
        for (int i = 0; i < 2; ++i)
            if (cudaStreamWaitEvent(p->lanes[i], p->ev_fork, 0) != cudaSuccess)
                return fail(ZLFFT_ERR_CUDA, "stream wait failed");
    }
    const cudaStream_t caller = st;
    const size_t quarter = p->scratch_bytes / 4;
    const bool gather = a.gin0 != nullptr;
    for (long long b0 = 0, ci = 0; b0 < a.batch; b0 += (long long)p->chunk, ++ci) {
        const long long nb = std::min<long long>((long long)p->chunk, a.batch - b0);
        if (fork) st = p->lanes[ci & 1];
        s0 = static_cast<char*>(p->d_scratch) + (size_t)(fork ? (ci & 1) : 0) * 2 * quarter;
        s1 = s0 + quarter;
        // this chunk's user buffers: base + stride, or the chunk's slice of the gather arrays
        const char* ui0 = gather ? nullptr : static_cast<const char*>(a.in0) + b0 * a.in_stride * in_elem;
        const char* ui1 = (!gather && a.in1) ? static_cast<const char*>(a.in1) + b0 * a.in_stride * in_elem : nullptr;
        char* uo0 = gather ? nullptr
                           : static_cast<char*>(a.out0) + b0 * a.out_stride * (dop == zlfft::kR2CSqrMag ? p->esize : out_elem);
        char* uo1 = (!gather && a.out1) ? static_cast<char*>(a.out1) + b0 * a.out_stride * out_elem : nullptr;
        const void* const* gi0 = gather ? a.gin0 + b0 : nullptr;
        const void* const* gi1 = (gather && a.gin1) ? a.gin1 + b0 : nullptr;
        void* const* go0 = gather ? a.gout0 + b0 : nullptr;
        void* const* go1 = (gather && a.gout1) ? a.gout1 + b0 : nullptr;
        cudaError_t e;
        // CFFT source/destination for this chunk
        const void* src0 = ui0;
        const void* src1 = ui1;
        long long src_stride = a.in_stride;
        int src_layout = il;
        if (c2r) {
            e = p->prec == ZLFFT_F32 ? launch_pre<float>(p, in_layout, ui0, ui1, s0, nb, a.in_stride, st, ctx, gi0, gi1)
                                     : launch_pre<double>(p, in_layout, ui0, ui1, s0, nb, a.in_stride, st, ctx, gi0, gi1);
            if (e != cudaSuccess) return cuda_fail(e, "rfft pre-step launch");
            src0 = s0;
            src1 = nullptr;
            src_stride = n;
            src_layout = ZLFFT_AOS;
        }
        char* bufs[2] = {c2r ? s1 : s0, c2r ? s0 : s1};
        bool split_done = false;
        for (int pi = 0; pi < np; ++pi) {
            const bool last = (pi + 1 == np);
            const bool gfirst = gather && pi == 0 && !c2r;  // the first pass reads gathered inputs
            zlfft::PassArgs pa{};
            pa.in0 = src0;
            pa.in1 = src1;
            pa.in_stride = src_stride;
            pa.batch = nb;
            pa.tws = p->d_tws;
            pa.tw = p->d_tw;
            pa.tctw = p->d_tctw ? static_cast<const char*>(p->d_tctw) + p->tctw_off[pi] * 2 * p->esize : nullptr;
            pa.err = p->d_err;
            pa.tma_out = (p->store_tma < 0 ? p->prec == ZLFFT_F32 : p->store_tma == 1) ? 1 : 0;
            pa.discard_in = (l2_discard_enabled() && (pi > 0 || c2r)) ? 1 : 0;  // the input is dead scratch
            if (gfirst) {
                pa.gin0 = gi0;
                pa.gin1 = gi1;
            }
            {
                // bulk-copy rows need 16-byte aligned sources (bases and transform stride)
                const size_t eb = (pi == 0 && src_layout == ZLFFT_SOA) ? p->esize : cx;
                pa.tma = (p->use_tma && !gfirst && aligned(src0, 16) && (!src1 || aligned(src1, 16)) &&
                          (nb == 1 || ((size_t)src_stride * eb) % 16 == 0)) ? 1 : 0;
                if (gfirst && a.gmaps) {  // gathered: the transforms' own maps, made with the batch
                    pa.gmaps = static_cast<const CUtensorMap*>(a.gmaps) + b0;
                    pa.tma = p->use_tma ? 1 : 0;
                }
            }
            // RFFT forward: the last pass fuses the split and writes the bins
            zlfft::PassLaunchFn split_fn = nullptr;
            if (p->fuse_split && last && r2c && !p->tc_form) {
                split_fn = pass_table(p).split[P - zlfft::kPassMinP][dop == zlfft::kR2CSqrMag ? 1 : 0][out_layout];
            }
            if ((last && !r2c) || split_fn) {
                pa.out0 = uo0;
                pa.out1 = uo1;
                pa.out_stride = a.out_stride;
                pa.gout0 = go0;
                pa.gout1 = go1;
                pa.rw = p->d_rw;
            } else {
                pa.out0 = bufs[pi & 1];
                pa.out1 = nullptr;
                pa.out_stride = n;
            }
            const int li = pi == 0 ? src_layout : ZLFFT_AOS;
            const int lo = (last && !r2c) ? ol : ZLFFT_AOS;
            zlfft::PassLaunchFn fn = split_fn ? split_fn : pick_pass(p, pi, fwd, li, lo);
            if (!fn) return fail(ZLFFT_ERR_UNSUPPORTED, "no pass kernel for order %d", p->order);
            e = fn(pa, st, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "pass launch");
            src0 = pa.out0;
            src1 = nullptr;
            src_stride = n;
            if (split_fn) split_done = true;
        }
        if (r2c && !split_done) {
            e = p->prec == ZLFFT_F32
                    ? launch_split<float>(p, dop, out_layout, src0, uo0, uo1, nb, a.out_stride, st, ctx, go0, go1)
                    : launch_split<double>(p, dop, out_layout, src0, uo0, uo1, nb, a.out_stride, st, ctx, go0, go1);
            if (e != cudaSuccess) return cuda_fail(e, "rfft split launch");
        }
    }
    if (fork) {
        for (int i = 0; i < 2; ++i) {
            if (cudaEventRecord(p->ev_join[i], p->lanes[i]) != cudaSuccess ||
                cudaStreamWaitEvent(caller, p->ev_join[i], 0) != cudaSuccess)
                return fail(ZLFFT_ERR_CUDA, "stream join failed");
        }
    }
    return ZLFFT_OK;
}

// FP32 complex order 14 (CFFT order 14, RFFT of real order 15) runs as one
// tile per transform, one pass over HBM. RFFT: the split fused, against two
// passes and a split kernel (+18-26% measured). CFFT: the next transform's
// input lands in the exchange buffer while the last group computes (plain
// +4%, fast form on par with its two passes) and no scratch is needed. The
// tensor-core form keeps its multi-pass passes.
bool tile14(const zlfft_plan_s* p) {
    return p->cfft_order == 14 && p->prec == ZLFFT_F32 && !p->tc_form;
}

// Argument checks shared by the device entry points (zlfft_exec_device and
// zlfft_exec_device_noalloc), and the kernel arguments they lead to. *a is
// filled only when the call has work (rc 0 and batch > 0).
int prepare_device_call(zlfft_plan_s* p, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                        void* out0, void* out1, size_t batch, size_t in_stride, size_t out_stride,
                        zlfft::TileArgs* a) {
    int rc = validate_op(p, op, in_layout, out_layout);
    if (rc) return rc;
    const Extents ex = extents(p, op);
    const bool in_soa = ex.in_complex && in_layout == ZLFFT_SOA;
    const bool out_soa = ex.out_complex && out_layout == ZLFFT_SOA;
    if (!in0 || (in_soa && !in1)) return fail(ZLFFT_ERR_INVALID_ARG, "null input pointer");
    if (!out0 || (out_soa && !out1)) return fail(ZLFFT_ERR_INVALID_ARG, "null output pointer");
    if (in_stride == 0) in_stride = ex.in_elems;
    if (out_stride == 0) out_stride = ex.out_elems;
    if (batch > 1 && (in_stride < ex.in_elems || out_stride < ex.out_elems))
        return fail(ZLFFT_ERR_INVALID_ARG, "stride smaller than one transform");
    // Alignment: AoS complex buffers are read as 8/16-byte vectors; an RFFT
    // real input is read as complex pairs, so it needs pair alignment and an
    // even stride; an RFFT real output is written as pairs likewise.
    const size_t pair = 2 * p->esize;
    const bool in_pairs = ex.in_complex ? !in_soa : (op != ZLFFT_BACKWARD);
    const bool out_pairs = ex.out_complex ? !out_soa : (p->kind == ZLFFT_R2C && op == ZLFFT_BACKWARD);
    if (in_pairs && !aligned(in0, pair)) return fail(ZLFFT_ERR_ALIGNMENT, "input must be %zu-byte aligned", pair);
    if (out_pairs && !aligned(out0, pair)) return fail(ZLFFT_ERR_ALIGNMENT, "output must be %zu-byte aligned", pair);
    if (!aligned(in0, p->esize) || (in1 && !aligned(in1, p->esize)) || !aligned(out0, p->esize) ||
        (out1 && !aligned(out1, p->esize)))
        return fail(ZLFFT_ERR_ALIGNMENT, "buffers must be aligned to the element type");
    if (!ex.in_complex && (in_stride % 2)) return fail(ZLFFT_ERR_INVALID_ARG, "RFFT real input stride must be even");
    if (p->kind == ZLFFT_R2C && op == ZLFFT_BACKWARD && (out_stride % 2))
        return fail(ZLFFT_ERR_INVALID_ARG, "RFFT real output stride must be even");
    if (p->kind == ZLFFT_C2C && in0 == out0 && in_layout != out_layout)
        return fail(ZLFFT_ERR_INVALID_ARG, "in-place transform needs the same layout on both sides");
    rc = check_aliasing(p, ex, in_soa, out_soa, in0, in1, out0, out1, batch, in_stride, out_stride);
    if (rc) return rc;
    if (batch == 0) return ZLFFT_OK;

    *a = zlfft::TileArgs{};
    a->in0 = in0;
    a->in1 = in_soa ? in1 : nullptr;
    a->out0 = out0;
    a->out1 = out_soa ? out1 : nullptr;
    a->batch = (long long)batch;
    // Strides in units of the element each kernel indexes: real sides of an
    // RFFT are indexed as complex pairs, except the squared-magnitude output.
    a->in_stride = (long long)(ex.in_complex ? in_stride : in_stride / 2);
    a->out_stride = (long long)((ex.out_complex || op == ZLFFT_FORWARD_SQR_MAG) ? out_stride : out_stride / 2);
    a->tw = p->d_tw;
    a->tws = p->d_tws;
    a->rw = p->d_rw;
    a->err = p->d_err;
    // Bulk (TMA) copies need 16-byte aligned sources: the bases and the
    // per-transform stride in bytes. The kernel reads directly otherwise.
    {
        const size_t in_elem_bytes = in_soa ? p->esize : 2 * p->esize;  // complex or pairs of reals
        const bool al = aligned(in0, 16) && (!in_soa || aligned(in1, 16)) &&
                        (batch == 1 || ((size_t)a->in_stride * in_elem_bytes) % 16 == 0);
        a->tma = (al && p->use_tma) ? 1 : 0;
    }
    // backward RFFT tiles stage their bins by cp.async: element alignment suffices
    if (device_op_code(p, op) == zlfft::kC2RBwd) a->tma = p->use_tma ? 1 : 0;
    return ZLFFT_OK;
}

// Intermediate buffers of one macro-path execution: chunks of `chunk`
// transforms alternate between `lanes` pipelines; pipeline i owns buf[i][0]
// and buf[i][1] (each `chunk` transforms long) and runs on stream[i] (lanes
// == 1: the caller's stream).
struct MacroScratch {
    char* buf[2][2];
    long long chunk;
    int lanes;
    cudaStream_t stream[2];
};

// The reference's macro path (zlfft_macro.cuh) over a batch: for each chunk,
// [RFFT backward pre-step] -> DIF pass(es) -> segment FFTs with the
// transposed store -> [RFFT forward split]. The DIF stages of one transform
// run in one pass up to 5 stages (1024-point units), else in two passes.
int exec_macro(zlfft_plan_s* p, int dop, int in_layout, int out_layout, const zlfft::TileArgs& a, cudaStream_t st,
               const zlfft::LaunchCtx& ctx, const MacroScratch& sc) {
    const int O = p->cfft_order, m = p->micro;
    const int nm = (O - m) / 2;
    const zlfft::MacroTable& t = p->prec == ZLFFT_F32 ? tables().m32 : tables().m64;
    int gp[2] = {nm, 0};
    int npass = 1;
    if (nm > zlfft::kMacroMaxG) {
        gp[0] = nm / 2;
        gp[1] = nm - nm / 2;
        npass = 2;
    }
    const size_t cx = 2 * p->esize;
    const long long n = 1LL << O;
    const bool fwd = (dop == zlfft::kC2CFwd || dop == zlfft::kR2CFwd || dop == zlfft::kR2CSqrMag);
    const bool r2c = (dop == zlfft::kR2CFwd || dop == zlfft::kR2CSqrMag);
    const bool c2r = (dop == zlfft::kC2RBwd);
    const int il = r2c ? ZLFFT_AOS : in_layout;   // R2C: real input read as complex pairs
    const int ol = c2r ? ZLFFT_AOS : out_layout;  // C2R: real output written as complex pairs
    const size_t in_elem = (in_layout == ZLFFT_SOA && !r2c) ? p->esize : cx;
    const size_t out_elem = (out_layout == ZLFFT_SOA && !c2r) ? p->esize : cx;
    for (long long b0 = 0, ci = 0; b0 < a.batch; b0 += sc.chunk, ++ci) {
        const long long nb = std::min<long long>(sc.chunk, a.batch - b0);
        const int lane = (int)(ci % sc.lanes);
        const cudaStream_t s = sc.lanes > 1 ? sc.stream[lane] : st;
        char* const* buf = sc.buf[lane];
        const char* ui0 = static_cast<const char*>(a.in0) + b0 * a.in_stride * in_elem;
        const char* ui1 = a.in1 ? static_cast<const char*>(a.in1) + b0 * a.in_stride * in_elem : nullptr;
        char* uo0 = static_cast<char*>(a.out0) + b0 * a.out_stride * (dop == zlfft::kR2CSqrMag ? p->esize : out_elem);
        char* uo1 = a.out1 ? static_cast<char*>(a.out1) + b0 * a.out_stride * out_elem : nullptr;
        cudaError_t e;
        const void* src0 = ui0;
        const void* src1 = ui1;
        long long src_stride = a.in_stride;
        int src_layout = il;
        int next = 0;  // the scratch buffer the next kernel writes
        if (c2r) {
            e = p->prec == ZLFFT_F32 ? launch_pre<float>(p, in_layout, ui0, ui1, buf[0], nb, a.in_stride, s, ctx)
                                     : launch_pre<double>(p, in_layout, ui0, ui1, buf[0], nb, a.in_stride, s, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "rfft pre-step launch");
            src0 = buf[0];
            src1 = nullptr;
            src_stride = n;
            src_layout = ZLFFT_AOS;
            next = 1;
        }
        int i0 = 0;
        for (int pi = 0; pi < npass; ++pi) {
            const int G = gp[pi];
            const bool last = (pi + 1 == npass);
            zlfft::DifArgs da{};
            da.in0 = src0;
            da.in1 = src1;
            da.out = buf[next];
            da.batch = nb;
            da.in_stride = src_stride;
            da.out_stride = n;
            da.tws = p->d_tws;
            da.order = O;
            da.i0 = i0;
            da.wlog = O - 2 * (i0 + G);
            da.nm = nm;
            da.mlog = m;
            const zlfft::DifLaunchFn fn =
                pi == 0 ? t.first[G - 1][fwd ? 1 : 0][src_layout][last ? 1 : 0] : t.mid[G - 1][last ? 1 : 0];
            e = fn(da, s, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "DIF pass launch");
            src0 = buf[next];
            src1 = nullptr;
            src_stride = n;
            next ^= 1;
            i0 += G;
        }
        // segment FFTs + transposed store: to the output, or (RFFT forward) to scratch for the split
        zlfft::SegArgs sa{};
        sa.t.in0 = src0;
        sa.t.batch = nb << (2 * nm);
        sa.t.in_stride = 1LL << m;
        sa.t.out_stride = 1LL << m;
        sa.t.tw = p->d_mtw;
        sa.t.tws = p->d_mtws;
        sa.t.err = p->d_err;
        sa.t.tma = p->use_tma;  // the scratch columns are 16-byte aligned and 2^m points long
        sa.slog = 2 * nm;
        if (r2c) {
            sa.out0 = buf[next];
            sa.out1 = nullptr;
            sa.out_stride = n;
        } else {
            sa.out0 = uo0;
            sa.out1 = uo1;
            sa.out_stride = a.out_stride;
        }
        sa.t.out0 = sa.out0;
        const zlfft::SegLaunchFn sfn = t.seg[m - zlfft::kSegMinM][fwd ? 1 : 0][r2c ? ZLFFT_AOS : ol];
        e = sfn(sa, s, ctx);
        if (e != cudaSuccess) return cuda_fail(e, "segment launch");
        if (r2c) {
            e = p->prec == ZLFFT_F32
                    ? launch_split<float>(p, dop, out_layout, buf[next], uo0, uo1, nb, a.out_stride, s, ctx)
                    : launch_split<double>(p, dop, out_layout, buf[next], uo0, uo1, nb, a.out_stride, s, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "rfft split launch");
        }
    }
    return ZLFFT_OK;
}

// exec_macro with the plan's scratch: chunks alternate between the plan's two
// internal streams, forked from and joined back to the caller's stream.
int exec_macro_planned(zlfft_plan_s* p, int dop, int in_layout, int out_layout, const zlfft::TileArgs& a,
                       cudaStream_t st, const zlfft::LaunchCtx& ctx) {
    int rc = ensure_scratch(p);
    if (rc) return rc;
    const size_t quarter = p->scratch_bytes / 4;
    MacroScratch sc{};
    for (int i = 0; i < 2; ++i) {
        sc.buf[i][0] = static_cast<char*>(p->d_scratch) + (size_t)i * 2 * quarter;
        sc.buf[i][1] = sc.buf[i][0] + quarter;
        sc.stream[i] = p->lanes[i];
    }
    sc.chunk = (long long)p->chunk;
    const long long nchunks = (a.batch + sc.chunk - 1) / sc.chunk;
    sc.lanes = (nchunks > 1 && p->nlanes > 1) ? 2 : 1;
    if (sc.lanes > 1) {
        if (cudaEventRecord(p->ev_fork, st) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "event record failed");
        for (int i = 0; i < 2; ++i)
            if (cudaStreamWaitEvent(p->lanes[i], p->ev_fork, 0) != cudaSuccess)
                return fail(ZLFFT_ERR_CUDA, "stream wait failed");
    }
    rc = exec_macro(p, dop, in_layout, out_layout, a, st, ctx, sc);
    if (rc) return rc;
    if (sc.lanes > 1) {
        for (int i = 0; i < 2; ++i) {
            if (cudaEventRecord(p->ev_join[i], p->lanes[i]) != cudaSuccess ||
                cudaStreamWaitEvent(st, p->ev_join[i], 0) != cudaSuccess)
                return fail(ZLFFT_ERR_CUDA, "stream join failed");
        }
    }
    return ZLFFT_OK;
}

// The kernels of one prepared device call (prepare_device_call), by size:
// the macro path, the multi-pass pipeline or one tile kernel launch.
int dispatch_device(zlfft_plan_s* p, int op, int in_layout, int out_layout, const zlfft::TileArgs& a,
                    cudaStream_t stream) {
    const int dop = device_op_code(p, op);
    const int P = p->cfft_order;
    zlfft::LaunchCtx ctx{p->num_sms, &p->launches};
    if (p->micro >= 0) {
        DeviceGuard g(p->device);
        return exec_macro_planned(p, dop, in_layout, out_layout, a, stream, ctx);
    }
    if (P > zlfft::kTileMaxP && !tile14(p)) {
        DeviceGuard g(p->device);
        return exec_multipass(p, dop, in_layout, out_layout, a, stream, ctx);
    }
    const zlfft::TileTable& t = p->prec == ZLFFT_F32 ? tables().f32 : tables().f64;
    zlfft::TileLaunchFn fn = t.fn[P][dop][in_layout][out_layout];
    if (p->fast_form && in_layout == ZLFFT_AOS && t.fast[P][dop][out_layout]) fn = t.fast[P][dop][out_layout];
    if (!fn) return fail(ZLFFT_ERR_UNSUPPORTED, "no kernel for this configuration");
    DeviceGuard g(p->device);
    cudaError_t e = fn(a, stream, ctx);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return ZLFFT_OK;
}

int exec_device_impl(zlfft_plan_s* p, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                     void* out0, void* out1, size_t batch, size_t in_stride, size_t out_stride, cudaStream_t stream) {
    zlfft::TileArgs a{};
    int rc = prepare_device_call(p, op, in_layout, out_layout, in0, in1, out0, out1, batch, in_stride, out_stride, &a);
    if (rc || batch == 0) return rc;
    return dispatch_device(p, op, in_layout, out_layout, a, stream);
}

// ------------------------------------------------------------------ STFT front end
// Frames f = 0..n_frames-1 of a real signal, frame f = signal[f*hop + n] *
// window[n] (n < N), each through the RFFT forward (bins or squared
// magnitudes), in one launch of the tile kernel: the frames are read straight
// from the signal (overlapping reads at stride hop) and windowed as they are
// loaded, so no framed or windowed copy is ever written.
int stft_impl(zlfft_plan_s* p, int op, int out_layout, const void* signal, size_t hop, const void* window,
              void* out0, void* out1, size_t n_frames, size_t out_stride, cudaStream_t stream) {
    if (p->kind != ZLFFT_R2C) return fail(ZLFFT_ERR_INVALID_ARG, "the STFT needs an RFFT plan");
    if (p->micro >= 0)
        return fail(ZLFFT_ERR_UNSUPPORTED, "the STFT runs the micro-only form; this plan follows the macro path");
    if (op != ZLFFT_FORWARD && op != ZLFFT_FORWARD_SQR_MAG)
        return fail(ZLFFT_ERR_INVALID_ARG, "STFT op must be FORWARD or FORWARD_SQR_MAG");
    if (out_layout != ZLFFT_AOS && out_layout != ZLFFT_SOA) return fail(ZLFFT_ERR_INVALID_ARG, "invalid layout");
    const int max_pc = p->prec == ZLFFT_F32 ? zlfft::kTileMaxP_f32 : zlfft::kTileMaxP_f64;
    if (p->cfft_order > max_pc) return fail(ZLFFT_ERR_UNSUPPORTED, "STFT frames up to order %d", max_pc + 1);
    if (hop == 0 || hop % 2) return fail(ZLFFT_ERR_INVALID_ARG, "hop must be even and positive (frames are read as pairs)");
    const bool soa = op == ZLFFT_FORWARD && out_layout == ZLFFT_SOA;
    if (!signal || !out0 || (soa && !out1)) return fail(ZLFFT_ERR_INVALID_ARG, "null buffer pointer");
    const size_t pair = 2 * p->esize;
    if (!aligned(signal, pair) || (window && !aligned(window, pair)))
        return fail(ZLFFT_ERR_ALIGNMENT, "signal and window must be %zu-byte aligned", pair);
    if (!aligned(out0, op == ZLFFT_FORWARD && !soa ? pair : p->esize) || (soa && !aligned(out1, p->esize)))
        return fail(ZLFFT_ERR_ALIGNMENT, "outputs must be aligned to their element type");
    const size_t nb = (size_t{1} << p->order) / 2 + 1;
    if (out_stride == 0) out_stride = nb;
    if (n_frames > 1 && out_stride < nb) return fail(ZLFFT_ERR_INVALID_ARG, "output stride smaller than one frame");
    if (n_frames == 0) return ZLFFT_OK;
    zlfft::TileArgs a{};
    a.in0 = signal;
    a.out0 = out0;
    a.out1 = soa ? out1 : nullptr;
    a.batch = (long long)n_frames;
    a.in_stride = (long long)(hop / 2);  // in complex pairs
    a.out_stride = (long long)out_stride;
    a.tw = p->d_tw;
    a.tws = p->d_tws;
    a.rw = p->d_rw;
    a.err = p->d_err;
    a.win = window;
    a.tma = (p->use_tma && aligned(signal, 16) && (n_frames == 1 || (hop * p->esize) % 16 == 0)) ? 1 : 0;
    const int dop = op == ZLFFT_FORWARD ? zlfft::kR2CFwd : zlfft::kR2CSqrMag;
    const zlfft::TileTable& t = p->prec == ZLFFT_F32 ? tables().f32 : tables().f64;
    zlfft::TileLaunchFn fn = window ? t.stft[p->cfft_order][op == ZLFFT_FORWARD ? 0 : 1][soa ? ZLFFT_SOA : ZLFFT_AOS]
                                    : t.fn[p->cfft_order][dop][ZLFFT_AOS][soa ? ZLFFT_SOA : ZLFFT_AOS];
    if (!fn) return fail(ZLFFT_ERR_UNSUPPORTED, "no kernel for this configuration");
    zlfft::LaunchCtx ctx{p->num_sms, &p->launches};
    DeviceGuard g(p->device);
    cudaError_t e = fn(a, stream, ctx);
    if (e != cudaSuccess) return cuda_fail(e, "STFT launch");
    return ZLFFT_OK;
}

// Inverse STFT / overlap-add (zlfft_istft.cuh): validation and dispatch.
int istft_impl(zlfft_plan_s* p, int in_layout, const void* in0, const void* in1, size_t in_stride, const void* filter,
               const void* window, size_t hop, size_t n_frames, void* signal, cudaStream_t stream) {
    if (p->kind != ZLFFT_R2C) return fail(ZLFFT_ERR_INVALID_ARG, "the inverse STFT needs an RFFT plan");
    if (p->micro >= 0)
        return fail(ZLFFT_ERR_UNSUPPORTED,
                    "the inverse STFT runs the micro-only form; this plan follows the macro path");
    if (in_layout != ZLFFT_AOS && in_layout != ZLFFT_SOA) return fail(ZLFFT_ERR_INVALID_ARG, "invalid layout");
    const zlfft::IstftTable& t = p->prec == ZLFFT_F32 ? tables().i32 : tables().i64;
    const int pc = p->cfft_order;
    zlfft::IstftLaunchFn fn = (pc >= 0 && pc <= zlfft::kTileMaxP) ? t.fn[pc][in_layout] : nullptr;
    if (!fn)
        return fail(ZLFFT_ERR_UNSUPPORTED, "inverse STFT frame orders are 10-%d for this precision",
                    p->prec == ZLFFT_F32 ? 14 : 13);
    const size_t n = size_t{1} << p->order;  // frame length in reals
    if (hop == 0 || hop % 2 || n % hop) return fail(ZLFFT_ERR_INVALID_ARG, "hop must be even and divide the frame length");
    const bool soa = in_layout == ZLFFT_SOA;
    if (!in0 || (soa && !in1) || !signal) return fail(ZLFFT_ERR_INVALID_ARG, "null buffer pointer");
    const size_t pair = 2 * p->esize;
    if (!aligned(in0, soa ? p->esize : pair) || (soa && !aligned(in1, p->esize)))
        return fail(ZLFFT_ERR_ALIGNMENT, "bins must be aligned to their element type");
    if ((filter && !aligned(filter, pair)) || (window && !aligned(window, pair)) || !aligned(signal, pair))
        return fail(ZLFFT_ERR_ALIGNMENT, "filter, window and signal must be %zu-byte aligned", pair);
    const size_t nb = n / 2 + 1;
    if (in_stride == 0) in_stride = nb;
    if (n_frames > 1 && in_stride < nb) return fail(ZLFFT_ERR_INVALID_ARG, "input stride smaller than one frame");
    if (n_frames == 0) return ZLFFT_OK;
    zlfft::TileArgs a{};
    a.in0 = in0;
    a.in1 = soa ? in1 : nullptr;
    a.batch = (long long)n_frames;
    a.in_stride = (long long)in_stride;
    a.out_stride = 0;
    a.tw = p->d_tw;
    a.tws = p->d_tws;
    a.rw = p->d_rw;
    a.err = p->d_err;
    zlfft::IstftArgs o{};
    o.filt = filter;
    o.win = window;
    o.sig = signal;
    o.n_frames = (long long)n_frames;
    o.hop = (long long)hop;
    o.k = (int)(n / hop);
    o.blocks = (long long)n_frames + o.k - 1;
    zlfft::LaunchCtx ctx{p->num_sms, &p->launches};
    DeviceGuard g(p->device);
    cudaError_t e = fn(a, o, stream, ctx);
    if (e != cudaSuccess) return cuda_fail(e, "inverse STFT launch");
    return ZLFFT_OK;
}

// ------------------------------------------------------------------ allocation-free execution
// Some callers cannot allocate device memory at the moment they run a
// transform: a real-time audio callback must not block on the allocator,
// and hosts that hand the whole device to a memory pool get no memory
// outside it. Orders 14 and up need intermediate buffers between their
// passes, which zlfft_exec_device allocates on first use. For those callers
// the library carries its own scratch: one array in device memory, reserved
// when the library's device code is loaded and held until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t{64} << 20;  // two halves of 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocSlot {
    std::mutex mu;
    void* ptr = nullptr;  // set once the lookup has succeeded
};
NoAllocSlot g_noalloc_slots[kNoAllocMaxDevices];

// Device address of the array on `device`. In host code the array's name is
// only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress, with that device current, on the first call that
// succeeds; a failed lookup is reported and tried again by the next call.
int noalloc_scratch(int device, void** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(ZLFFT_ERR_INVALID_ARG, "device %d out of range", device);
    NoAllocSlot& slot = g_noalloc_slots[device];
    std::lock_guard<std::mutex> lock(slot.mu);
    if (!slot.ptr) {
        DeviceGuard g(device);
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        slot.ptr = ptr;
    }
    *out = slot.ptr;
    return ZLFFT_OK;
}

// The largest order of the plan's kind and precision whose transform fits
// one half of the array (an RFFT's inner CFFT is one order below it).
int noalloc_max_order(const zlfft_plan_s* p) {
    int o = 0;
    while ((size_t{1} << (o + 1)) * 2 * p->esize <= kNoAllocScratchBytes / 2) ++o;
    return p->kind == ZLFFT_R2C ? o + 1 : o;
}

// The multi-pass orders with the built-in array as the pass intermediates:
// chunks of transforms, one after another on the caller's stream (no helper
// streams or events are created). Same kernels and arithmetic as
// exec_multipass.
int exec_multipass_noalloc(zlfft_plan_s* p, int dop, int in_layout, int out_layout, const zlfft::TileArgs& a,
                           cudaStream_t st, const zlfft::LaunchCtx& ctx) {
    const int P = p->cfft_order;
    if (P < zlfft::kPassMinP || P > zlfft::kPassMaxP)
        return fail(ZLFFT_ERR_UNSUPPORTED, "order %d is above the supported maximum", p->order);
    const size_t cx = 2 * p->esize;
    const long long n = 1LL << P;
    const size_t half = kNoAllocScratchBytes / 2;
    const size_t per = (size_t)n * cx;
    if (per > half)
        return fail(ZLFFT_ERR_UNSUPPORTED,
                    "one transform needs %zu bytes of intermediate buffer; the allocation-free entry point holds "
                    "%zu per buffer (order <= %d for this kind and precision)",
                    per, half, noalloc_max_order(p));
    void* base = nullptr;
    int rc = noalloc_scratch(p->device, &base);
    if (rc) return rc;
    const long long chunk = (long long)(half / per);
    char* s0 = static_cast<char*>(base);
    char* s1 = s0 + half;
    const zlfft::PassTable& t = pass_table(p);
    const auto& row = t.fn[P - zlfft::kPassMinP];
    int np = 0;
    while (np < zlfft::kMaxPasses && row[np][1][0][0]) ++np;
    const bool fwd = (dop == zlfft::kC2CFwd || dop == zlfft::kR2CFwd || dop == zlfft::kR2CSqrMag);
    const bool r2c = (dop == zlfft::kR2CFwd || dop == zlfft::kR2CSqrMag);
    const bool c2r = (dop == zlfft::kC2RBwd);
    const int il = r2c ? ZLFFT_AOS : in_layout;
    const int ol = c2r ? ZLFFT_AOS : out_layout;
    const size_t in_elem = (in_layout == ZLFFT_SOA && !r2c) ? p->esize : cx;
    const size_t out_elem = (out_layout == ZLFFT_SOA && !c2r) ? p->esize : cx;
    for (long long b0 = 0; b0 < a.batch; b0 += chunk) {
        const long long nb = std::min<long long>(chunk, a.batch - b0);
        const char* ui0 = static_cast<const char*>(a.in0) + b0 * a.in_stride * in_elem;
        const char* ui1 = a.in1 ? static_cast<const char*>(a.in1) + b0 * a.in_stride * in_elem : nullptr;
        char* uo0 = static_cast<char*>(a.out0) + b0 * a.out_stride * (dop == zlfft::kR2CSqrMag ? p->esize : out_elem);
        char* uo1 = a.out1 ? static_cast<char*>(a.out1) + b0 * a.out_stride * out_elem : nullptr;
        cudaError_t e;
        const void* src0 = ui0;
        const void* src1 = ui1;
        long long src_stride = a.in_stride;
        int src_layout = il;
        if (c2r) {
            e = p->prec == ZLFFT_F32 ? launch_pre<float>(p, in_layout, ui0, ui1, s0, nb, a.in_stride, st, ctx)
                                     : launch_pre<double>(p, in_layout, ui0, ui1, s0, nb, a.in_stride, st, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "rfft pre-step launch");
            src0 = s0;
            src1 = nullptr;
            src_stride = n;
            src_layout = ZLFFT_AOS;
        }
        char* bufs[2] = {c2r ? s1 : s0, c2r ? s0 : s1};
        for (int pi = 0; pi < np; ++pi) {
            const bool last = (pi + 1 == np);
            zlfft::PassArgs pa{};
            pa.in0 = src0;
            pa.in1 = src1;
            pa.in_stride = src_stride;
            pa.batch = nb;
            pa.tws = p->d_tws;
            pa.tw = p->d_tw;
            pa.tctw = p->d_tctw ? static_cast<const char*>(p->d_tctw) + p->tctw_off[pi] * 2 * p->esize : nullptr;
            pa.err = p->d_err;
            pa.tma_out = (p->store_tma < 0 ? p->prec == ZLFFT_F32 : p->store_tma == 1) ? 1 : 0;
            pa.discard_in = (l2_discard_enabled() && (pi > 0 || c2r)) ? 1 : 0;  // the input is dead scratch
            const size_t eb = (pi == 0 && src_layout == ZLFFT_SOA) ? p->esize : cx;
            pa.tma = (p->use_tma && aligned(src0, 16) && (!src1 || aligned(src1, 16)) &&
                      (nb == 1 || ((size_t)src_stride * eb) % 16 == 0)) ? 1 : 0;
            if (last && !r2c) {
                pa.out0 = uo0;
                pa.out1 = uo1;
                pa.out_stride = a.out_stride;
            } else {
                pa.out0 = bufs[pi & 1];
                pa.out1 = nullptr;
                pa.out_stride = n;
            }
            const int li = pi == 0 ? src_layout : ZLFFT_AOS;
            const int lo = (last && !r2c) ? ol : ZLFFT_AOS;
            zlfft::PassLaunchFn fn = pick_pass(p, pi, fwd, li, lo);
            if (!fn) return fail(ZLFFT_ERR_UNSUPPORTED, "no pass kernel for order %d", p->order);
            e = fn(pa, st, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "pass launch");
            src0 = pa.out0;
            src1 = nullptr;
            src_stride = n;
        }
        if (r2c) {
            e = p->prec == ZLFFT_F32
                    ? launch_split<float>(p, dop, out_layout, src0, uo0, uo1, nb, a.out_stride, st, ctx)
                    : launch_split<double>(p, dop, out_layout, src0, uo0, uo1, nb, a.out_stride, st, ctx);
            if (e != cudaSuccess) return cuda_fail(e, "rfft split launch");
        }
    }
    return ZLFFT_OK;
}

// Argument checks of zlfft_exec_device, then the allocation-free dispatch:
// the single-CTA sizes run exactly as in zlfft_exec_device (they use no
// scratch); the multi-pass and macro-path sizes pass their intermediates
// through the built-in array.
int exec_device_noalloc_impl(zlfft_plan_s* p, int op, int in_layout, int out_layout, const void* in0,
                             const void* in1, void* out0, void* out1, size_t batch, size_t in_stride,
                             size_t out_stride, cudaStream_t stream) {
    if (p->micro < 0 && (p->cfft_order <= zlfft::kTileMaxP || tile14(p)))
        return exec_device_impl(p, op, in_layout, out_layout, in0, in1, out0, out1, batch, in_stride, out_stride,
                                stream);
    zlfft::TileArgs a{};
    int rc = prepare_device_call(p, op, in_layout, out_layout, in0, in1, out0, out1, batch, in_stride, out_stride, &a);
    if (rc || batch == 0) return rc;
    zlfft::LaunchCtx ctx{p->num_sms, &p->launches};
    DeviceGuard g(p->device);
    if (p->micro >= 0) {
        const size_t half = kNoAllocScratchBytes / 2;
        const size_t per = (size_t{1} << p->cfft_order) * 2 * p->esize;
        if (per > half)
            return fail(ZLFFT_ERR_UNSUPPORTED,
                        "one transform needs %zu bytes of intermediate buffer; the allocation-free entry point "
                        "holds %zu per buffer (order <= %d for this kind and precision)",
                        per, half, noalloc_max_order(p));
        void* base = nullptr;
        rc = noalloc_scratch(p->device, &base);
        if (rc) return rc;
        MacroScratch sc{};
        sc.buf[0][0] = static_cast<char*>(base);
        sc.buf[0][1] = sc.buf[0][0] + half;
        sc.chunk = (long long)(half / per);
        sc.lanes = 1;
        return exec_macro(p, device_op_code(p, op), in_layout, out_layout, a, stream, ctx, sc);
    }
    return exec_multipass_noalloc(p, device_op_code(p, op), in_layout, out_layout, a, stream, ctx);
}

int ensure_staging(zlfft_plan_s* p, size_t in_bytes, size_t out_bytes) {
    if (!p->ev_host && cudaEventCreateWithFlags(&p->ev_host, cudaEventDisableTiming) != cudaSuccess)
        return fail(ZLFFT_ERR_CUDA, "event creation failed");
    if (!p->h_err) {
        if (cudaMallocHost(reinterpret_cast<void**>(&p->h_err), sizeof(int)) != cudaSuccess)
            return alloc_fail("staging", sizeof(int));
        *p->h_err = 0;
    }
    if (in_bytes > p->stage_in_bytes) {
        if (p->h_in) cudaFreeHost(p->h_in);
        if (p->d_in) cudaFree(p->d_in);
        p->h_in = p->d_in = nullptr;
        p->stage_in_bytes = 0;
        if (cudaMallocHost(&p->h_in, in_bytes) != cudaSuccess || cudaMalloc(&p->d_in, in_bytes) != cudaSuccess)
            return alloc_fail("staging", in_bytes);
        p->stage_in_bytes = in_bytes;
    }
    if (out_bytes > p->stage_out_bytes) {
        if (p->h_out) cudaFreeHost(p->h_out);
        if (p->d_out) cudaFree(p->d_out);
        p->h_out = p->d_out = nullptr;
        p->stage_out_bytes = 0;
        if (cudaMallocHost(&p->h_out, out_bytes) != cudaSuccess || cudaMalloc(&p->d_out, out_bytes) != cudaSuccess)
            return alloc_fail("staging", out_bytes);
        p->stage_out_bytes = out_bytes;
    }
    return ZLFFT_OK;
}

bool is_pinned(const void* ptr) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Single small transforms from host buffers: the reference's own call
// pattern (one transform per call, often from an audio thread). Copies
// queued around the kernel cost more than the transform, so the kernel reads
// its input from, and writes its output to, page-locked host buffers mapped
// into the device's address space: a call copies the caller's input into the
// mapped buffer, launches one kernel, synchronises the plan's stream once and
// copies the output out. The kernel's error word is mapped as well, so no
// separate read-back is queued. Inputs are read with plain loads (no bulk
// copies from host memory). ZLFFT_HOST_ZEROCOPY=0 turns the path off
// (comparison with the staged path).
constexpr size_t kSmallHostBytes = 256 << 10;  // in + out bytes of one transform, at most

bool small_host_call(const zlfft_plan_s* p, size_t batch, size_t in_bytes, size_t out_bytes) {
    static const bool enabled = [] {
        const char* e = getenv("ZLFFT_HOST_ZEROCOPY");
        return !(e && e[0] == '0');
    }();
    return enabled && batch == 1 && p->micro < 0 && p->cfft_order <= zlfft::kTileMaxP &&
           in_bytes + out_bytes <= kSmallHostBytes;
}

int ensure_mapped(zlfft_plan_s* p, size_t in_bytes, size_t out_bytes) {
    auto grow = [](void** buf, size_t* have, size_t want) -> bool {
        if (want <= *have) return true;
        if (*buf) cudaFreeHost(*buf);
        *buf = nullptr;
        *have = 0;
        if (cudaHostAlloc(buf, want, cudaHostAllocMapped) != cudaSuccess) return false;
        *have = want;
        return true;
    };
    if (!grow(&p->hm_in, &p->hm_in_bytes, in_bytes) || !grow(&p->hm_out, &p->hm_out_bytes, out_bytes))
        return alloc_fail("mapped staging", in_bytes + out_bytes);
    if (!p->hm_err) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&p->hm_err), sizeof(int), cudaHostAllocMapped) != cudaSuccess)
            return alloc_fail("mapped error word", sizeof(int));
        *p->hm_err = 0;
    }
    ZL_CUDA(cudaHostGetDevicePointer(&p->dm_in, p->hm_in, 0));
    ZL_CUDA(cudaHostGetDevicePointer(&p->dm_out, p->hm_out, 0));
    ZL_CUDA(cudaHostGetDevicePointer(&p->dm_err, p->hm_err, 0));
    return ZLFFT_OK;
}

int exec_host_small(zlfft_plan_s* p, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                    void* out0, void* out1, size_t in_part, size_t out_part, int in_parts, int out_parts) {
    if (in_part * in_parts > p->hm_in_bytes || out_part * out_parts > p->hm_out_bytes || !p->hm_err) {
        const int rc0 = ensure_mapped(p, in_part * in_parts, out_part * out_parts);
        if (rc0) return rc0;
    }
    memcpy(p->hm_in, in0, in_part);
    if (in_parts == 2) memcpy(static_cast<char*>(p->hm_in) + in_part, in1, in_part);
    char* di = static_cast<char*>(p->dm_in);
    char* dd = static_cast<char*>(p->dm_out);
    zlfft::TileArgs a{};
    int rc = prepare_device_call(p, op, in_layout, out_layout, di, in_parts == 2 ? di + in_part : nullptr, dd,
                                 out_parts == 2 ? dd + out_part : nullptr, 1, 0, 0, &a);
    if (rc) return rc;
    a.tma = 0;
    a.err = static_cast<int*>(p->dm_err);
    rc = dispatch_device(p, op, in_layout, out_layout, a, p->stream);
    if (rc) {
        cudaStreamSynchronize(p->stream);
        return rc;
    }
    ZL_CUDA(cudaStreamSynchronize(p->stream));
    const int e = *static_cast<volatile int*>(p->hm_err);
    if (e) {
        *p->hm_err = 0;
        return fail(ZLFFT_ERR_DEVICE_TIMEOUT, "a device-side wait ran out of its iteration limit (code %d)", e);
    }
    memcpy(out0, p->hm_out, out_part);
    if (out_parts == 2) memcpy(out1, static_cast<char*>(p->hm_out) + out_part, out_part);
    return ZLFFT_OK;
}

// Host-pointer path: H2D copy of the input (directly from the caller's
// buffer when it is page-locked, else through the plan's pinned staging),
// the device kernel on the plan's stream, D2H copy back, synchronise.
// The batch is cut into chunks so that the copies of one chunk overlap the
// kernel and the opposite-direction copy of its neighbours (two streams).
int exec_host_impl(zlfft_plan_s* p, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                   void* out0, void* out1, size_t batch) {
    int rc = validate_op(p, op, in_layout, out_layout);
    if (rc) return rc;
    const Extents ex = extents(p, op);
    const bool in_soa = ex.in_complex && in_layout == ZLFFT_SOA;
    const bool out_soa = ex.out_complex && out_layout == ZLFFT_SOA;
    if (!in0 || (in_soa && !in1) || !out0 || (out_soa && !out1))
        return fail(ZLFFT_ERR_INVALID_ARG, "null buffer pointer");
    if (batch == 0) return ZLFFT_OK;
    // bytes of one transform on each side, per part (SoA: per re/im array)
    const size_t in_part = ex.in_elems * (ex.in_complex && !in_soa ? 2 : 1) * p->esize;
    const size_t out_part = ex.out_elems * (ex.out_complex && !out_soa ? 2 : 1) * p->esize;
    const int in_parts = in_soa ? 2 : 1, out_parts = out_soa ? 2 : 1;
    const size_t in_bytes = in_part * in_parts * batch, out_bytes = out_part * out_parts * batch;
    std::lock_guard<std::mutex> lock(p->mu);
    DeviceGuard g(p->device);
    if (small_host_call(p, batch, in_bytes, out_bytes))
        return exec_host_small(p, op, in_layout, out_layout, in0, in1, out0, out1, in_part, out_part, in_parts,
                               out_parts);
    const bool pin_in = is_pinned(in0) && (!in_soa || is_pinned(in1));
    const bool pin_out = is_pinned(out0) && (!out_soa || is_pinned(out1));
    rc = ensure_staging(p, in_bytes, out_bytes);
    if (rc) return rc;
    // Device buffers: [part 0 of all transforms][part 1 of all transforms].
    char* din = static_cast<char*>(p->d_in);
    char* dout = static_cast<char*>(p->d_out);
    const void* src[2] = {in0, in1};
    void* dst[2] = {out0, out1};
    if (!pin_in) {
        for (int q = 0; q < in_parts; ++q)
            memcpy(static_cast<char*>(p->h_in) + q * in_part * batch, src[q], in_part * batch);
    }
    // Chunking: an eighth of the call's input, within 8-32 MiB, at least one
    // transform (ZLFFT_HOST_CHUNK_MB fixes the size). Measured from pinned
    // buffers: the 2 GiB CFFT<float> orders 14/16/20, forward + backward, 16 MiB
    // 87.9-88.5 GB/s, 32 MiB 92.1, 64 MiB 90.6 (three streams: no better);
    // CFFT<double> order 16 x 512 (512 MiB) 88.1 -> 89.7 from 16 to 32 MiB; but
    // RFFT<float> order 12 x 8192 (128 MiB) 79.1 -> 76.8, where fewer chunks
    // leave more of the first copy in and the last copy out unoverlapped.
    static const size_t chunk_env = [] {
        const char* e = getenv("ZLFFT_HOST_CHUNK_MB");
        const long v = e ? atol(e) : 0;
        return v > 0 ? (size_t)v << 20 : (size_t)0;
    }();
    const size_t in_total = in_part * in_parts * batch;
    const size_t chunk_bytes =
        chunk_env ? chunk_env : std::min<size_t>(std::max<size_t>(in_total / 8, size_t{8} << 20), size_t{32} << 20);
    constexpr int nss = 2;
    size_t chunk = chunk_bytes / (in_part * in_parts);
    if (chunk == 0) chunk = 1;
    if (chunk > batch) chunk = batch;
    // The chunks' copies alternate between two streams. Their transforms share
    // the plan's scratch (orders >= 14), so each one waits for the previous
    // chunk's (ev_host); the copies still overlap the neighbouring transforms.
    cudaStream_t ss[nss] = {p->stream, p->stream2};
    // on failure, let every copy already queued finish before returning, so
    // nothing touches the caller's buffers afterwards
    auto drain = [&](int code) {
        for (int i = 0; i < nss; ++i) cudaStreamSynchronize(ss[i]);
        return code;
    };
    for (size_t b0 = 0, c = 0; b0 < batch; b0 += chunk, ++c) {
        const size_t nb = (batch - b0 < chunk) ? batch - b0 : chunk;
        cudaStream_t st = ss[c % nss];
        for (int q = 0; q < in_parts; ++q) {
            const char* h = pin_in ? static_cast<const char*>(src[q]) : static_cast<const char*>(p->h_in) + q * in_part * batch;
            const cudaError_t e = cudaMemcpyAsync(din + q * in_part * batch + b0 * in_part, h + b0 * in_part,
                                                  nb * in_part, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return drain(cuda_fail(e, "cudaMemcpyAsync (H2D)"));
        }
        const void* i0 = din + b0 * in_part;
        const void* i1 = in_soa ? din + in_part * batch + b0 * in_part : nullptr;
        void* o0 = dout + b0 * out_part;
        void* o1 = out_soa ? dout + out_part * batch + b0 * out_part : nullptr;
        if (c > 0 && cudaStreamWaitEvent(st, p->ev_host, 0) != cudaSuccess)
            return drain(fail(ZLFFT_ERR_CUDA, "stream wait failed"));
        // dense strides: the device buffers hold whole transforms back to back
        rc = exec_device_impl(p, op, in_layout, out_layout, i0, i1, o0, o1, nb, 0, 0, st);
        if (rc) return drain(rc);
        if (cudaEventRecord(p->ev_host, st) != cudaSuccess) return drain(fail(ZLFFT_ERR_CUDA, "event record failed"));
        for (int q = 0; q < out_parts; ++q) {
            char* h = pin_out ? static_cast<char*>(dst[q]) : static_cast<char*>(p->h_out) + q * out_part * batch;
            const cudaError_t e = cudaMemcpyAsync(h + b0 * out_part, dout + q * out_part * batch + b0 * out_part,
                                                  nb * out_part, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return drain(cuda_fail(e, "cudaMemcpyAsync (D2H)"));
        }
    }
    // the error word comes back behind the last chunk's transform (the
    // chunks' transforms are ordered by ev_host), with the output copies
    {
        const cudaStream_t last = ss[(int)(((batch + chunk - 1) / chunk - 1) % nss)];
        const cudaError_t e = cudaMemcpyAsync(p->h_err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, last);
        if (e != cudaSuccess) return drain(cuda_fail(e, "cudaMemcpyAsync (error word)"));
    }
    for (int i = 0; i < nss; ++i) ZL_CUDA(cudaStreamSynchronize(ss[i]));
    if (const int derr = *static_cast<volatile int*>(p->h_err)) {
        *p->h_err = 0;
        cudaMemset(p->d_err, 0, sizeof(int));
        return fail(ZLFFT_ERR_DEVICE_TIMEOUT, "a device-side wait ran out of its iteration limit (code %d)", derr);
    }
    if (!pin_out) {
        for (int q = 0; q < out_parts; ++q)
            memcpy(dst[q], static_cast<char*>(p->h_out) + q * out_part * batch, out_part * batch);
    }
    return ZLFFT_OK;
}


// ------------------------------------------------------------------ mixed batches
// A mixed batch is sorted on the host into groups of one (precision, kind,
// order, operation); each group's transforms are addressed through gathered
// pointer arrays (transform t of the group reads gin[t], writes gout[t]).
// Groups of complex order 2..13 become tiles of persistent launches, one per
// (precision, order class): orders 2..11 in 128-thread CTAs, 12..13 in
// 512-thread CTAs (zlfft_mixed.cuh); the others run as gathered batched
// launches of the tile kernel (orders 0, 1 and the FP32 order-14 tile) or of
// the multi-pass pipeline (14 and up), largest first.
struct MixedGroupHost {
    zlfft_plan plan;
    int prec;
    int dop;     // device operation code
    int P;       // complex order
    size_t first;  // offset of the group in the gather arrays
    size_t count;
    const void* d_maps = nullptr;  // multi-pass groups: per-transform first-pass input maps, or null
    bool in_aligned = false;       // every input of the group is 16-byte aligned (bulk copies)
};

}  // namespace

struct zlfft_mixed_s {
    int device = 0;
    int num_sms = 0;
    std::vector<zlfft_plan> plans;
    std::vector<MixedGroupHost> groups;  // sorted by complex order, largest first
    void* d_mem = nullptr;               // gather arrays, group records, work lists, counters
    const void** d_gin = nullptr;
    void** d_gout = nullptr;
    zlfft::MixedGroup* d_mgroups[2] = {nullptr, nullptr};  // per precision
    zlfft::MixedItem* d_items[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [precision][order class]
    int n_items[2][2] = {{0, 0}, {0, 0}};
    int* d_counter = nullptr;  // one work-list counter per (precision, order class)
    cudaStream_t cap_stream = nullptr;
    // persistent schedule: the multi-pass and large-tile groups run on these
    // streams (forked from the caller's stream, joined back) beside the
    // persistent launch
    static constexpr int kSideStreams = 2;
    cudaStream_t side[kSideStreams] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[kSideStreams] = {nullptr, nullptr};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    size_t graph_launches = 0;  // kernels recorded in the graph
    std::atomic<size_t> launches{0};
    std::mutex mu;
};

namespace {

void mixed_release(zlfft_mixed m) {
    if (!m) return;
    {
        DeviceGuard g(m->device);
        if (m->graph_exec) cudaGraphExecDestroy(m->graph_exec);
        if (m->graph) cudaGraphDestroy(m->graph);
        if (m->cap_stream) cudaStreamDestroy(m->cap_stream);
        for (int i = 0; i < zlfft_mixed_s::kSideStreams; ++i) {
            if (m->side[i]) cudaStreamDestroy(m->side[i]);
            if (m->ev_join[i]) cudaEventDestroy(m->ev_join[i]);
        }
        if (m->ev_fork) cudaEventDestroy(m->ev_fork);
        if (m->d_mem) cudaFree(m->d_mem);
    }
    for (zlfft_plan p : m->plans) release(p);
    delete m;
}

int mixed_validate(const zlfft_desc& d, size_t i) {
    if (d.kind != ZLFFT_C2C && d.kind != ZLFFT_R2C)
        return fail(ZLFFT_ERR_INVALID_ARG, "descriptor %zu: invalid kind %d", i, d.kind);
    if (d.precision != ZLFFT_F32 && d.precision != ZLFFT_F64)
        return fail(ZLFFT_ERR_INVALID_ARG, "descriptor %zu: invalid precision %d", i, d.precision);
    const int lo = d.kind == ZLFFT_C2C ? 0 : 1;
    const int hi = zlfft::kPassMaxP + (d.kind == ZLFFT_C2C ? 0 : 1);
    if (d.order < lo || d.order > hi)
        return fail(ZLFFT_ERR_UNSUPPORTED, "descriptor %zu: order %d outside %d..%d", i, d.order, lo, hi);
    if (d.op < ZLFFT_FORWARD || d.op > ZLFFT_FORWARD_SQR_MAG)
        return fail(ZLFFT_ERR_INVALID_ARG, "descriptor %zu: invalid op %d", i, d.op);
    if (d.op == ZLFFT_FORWARD_SQR_MAG && d.kind != ZLFFT_R2C)
        return fail(ZLFFT_ERR_INVALID_ARG, "descriptor %zu: forward_sqr_mag is an RFFT operation", i);
    if (!d.in || !d.out) return fail(ZLFFT_ERR_INVALID_ARG, "descriptor %zu: null buffer pointer", i);
    const size_t es = d.precision == ZLFFT_F32 ? 4 : 8;
    // complex values and real inputs are accessed as pairs; the sqr_mag output as reals
    if (!aligned(d.in, 2 * es) || !aligned(d.out, d.op == ZLFFT_FORWARD_SQR_MAG ? es : 2 * es))
        return fail(ZLFFT_ERR_ALIGNMENT, "descriptor %zu: buffers must be %zu-byte aligned", i, 2 * es);
    return ZLFFT_OK;
}

// The transforms of a mixed batch run concurrently, in no fixed order. So no
// output may overlap another transform's output or input: the result would
// depend on the schedule, where the reference's calls, one after another,
// have one answer. Inputs may be shared, and a transform's output may overlap
// its own input (every kernel reads a transform's input before writing its
// output), which covers in place. O(n log n): outputs sorted by start must be
// disjoint; each input is then checked against the outputs around it.
int mixed_check_overlaps(const zlfft_desc* descs, size_t n) {
    struct Span {
        uintptr_t lo, hi;
        size_t i;
    };
    std::vector<Span> outs(n), ins(n);
    for (size_t i = 0; i < n; ++i) {
        const zlfft_desc& d = descs[i];
        const size_t es = d.precision == ZLFFT_F32 ? 4 : 8;
        const size_t N = size_t{1} << d.order, nb = N / 2 + 1;
        size_t ib, ob;
        if (d.kind == ZLFFT_C2C) {
            ib = ob = 2 * es * N;
        } else if (d.op == ZLFFT_BACKWARD) {
            ib = 2 * es * nb;
            ob = es * N;
        } else {
            ib = es * N;
            ob = d.op == ZLFFT_FORWARD ? 2 * es * nb : es * nb;
        }
        const uintptr_t in = reinterpret_cast<uintptr_t>(d.in), out = reinterpret_cast<uintptr_t>(d.out);
        ins[i] = Span{in, in + ib, i};
        outs[i] = Span{out, out + ob, i};
    }
    std::sort(outs.begin(), outs.end(), [](const Span& a, const Span& b) { return a.lo < b.lo; });
    for (size_t k = 0; k + 1 < n; ++k)
        if (outs[k].hi > outs[k + 1].lo)
            return fail(ZLFFT_ERR_INVALID_ARG,
                        "descriptors %zu and %zu: outputs overlap (the transforms of a batch run concurrently)",
                        outs[k].i, outs[k + 1].i);
    for (const Span& a : ins) {
        // outputs are disjoint and sorted, so their ends are sorted too
        auto it = std::upper_bound(outs.begin(), outs.end(), a.lo, [](uintptr_t v, const Span& o) { return v < o.hi; });
        for (; it != outs.end() && it->lo < a.hi; ++it)
            if (it->i != a.i)
                return fail(ZLFFT_ERR_INVALID_ARG,
                            "descriptor %zu writes over the input of descriptor %zu (the transforms of a batch run "
                            "concurrently)",
                            it->i, a.i);
    }
    return ZLFFT_OK;
}

// Cost of one persistent tile of complex order P (points x stages): orders
// 4 and up hold 128 * 16 points per tile, so the cost grows with P.
long long mixed_tile_cost(int P) { return (long long)zlfft::mixed_tpc(P) * (1LL << P) * (P > 0 ? P : 1); }

zlfft::TileArgs mixed_args(const zlfft_mixed_s* m, const MixedGroupHost& g) {
    zlfft::TileArgs a{};
    a.batch = (long long)g.count;
    a.tw = g.plan->d_tw;
    a.tws = g.plan->d_tws;
    a.rw = g.plan->d_rw;
    a.err = g.plan->d_err;
    // gathered tile launches stage their inputs by bulk copies from each pointer
    // (the forward operations; the persistent kernel and the passes decide for themselves)
    a.tma = (g.in_aligned && g.plan->use_tma && g.dop != zlfft::kC2RBwd) ? 1 : 0;
    a.gin0 = m->d_gin + g.first;
    a.gout0 = m->d_gout + g.first;
    a.gmaps = g.d_maps;
    return a;
}

bool mixed_in_persistent(const MixedGroupHost& g) { return g.P >= zlfft::kMixedMinP && g.P <= zlfft::kMixedTopP; }

// One group as its own batched launch(es) on `st`.
int mixed_run_group(zlfft_mixed_s* m, const MixedGroupHost& g, cudaStream_t st) {
    zlfft::LaunchCtx ctx{m->num_sms, &m->launches};
    const zlfft::TileArgs a = mixed_args(m, g);
    if (g.P > zlfft::kTileMaxP && !tile14(g.plan))
        return exec_multipass(g.plan, g.dop, ZLFFT_AOS, ZLFFT_AOS, a, st, ctx);
    const zlfft::GatherTable& t = g.prec == ZLFFT_F32 ? tables().g32 : tables().g64;
    zlfft::TileLaunchFn fn = t.fn[g.P][g.dop];
    if (g.plan->fast_form && t.fast[g.P][g.dop]) fn = t.fast[g.P][g.dop];  // the tuned plan's form
    if (!fn) return fail(ZLFFT_ERR_UNSUPPORTED, "no gathered kernel for order %d", g.P);
    cudaError_t e = fn(a, st, ctx);
    if (e != cudaSuccess) return cuda_fail(e, "gathered tile launch");
    return ZLFFT_OK;
}

int mixed_run(zlfft_mixed_s* m, int schedule, cudaStream_t st) {
    const bool persistent = schedule != ZLFFT_SCHED_PER_ORDER;
    if (!persistent) {  // the baseline: one batched launch (or pipeline) per group, in order
        for (const MixedGroupHost& g : m->groups) {
            int rc = mixed_run_group(m, g, st);
            if (rc) return rc;
        }
        return ZLFFT_OK;
    }
    // The groups outside the persistent kernel (largest first) are dealt to the
    // side streams, so groups of different orders overlap each other's tails
    // and the persistent launch on the caller's stream. The groups of one plan
    // (one size, several operations; adjacent in the sorted order) share its
    // scratch, so they are dealt to the same stream, one after another.
    int big = 0;
    for (const MixedGroupHost& g : m->groups) big += mixed_in_persistent(g) ? 0 : 1;
    if (big) {
        ZL_CUDA(cudaEventRecord(m->ev_fork, st));
        for (int i = 0; i < zlfft_mixed_s::kSideStreams; ++i) ZL_CUDA(cudaStreamWaitEvent(m->side[i], m->ev_fork, 0));
        int si = -1;
        const zlfft_plan_s* prev = nullptr;
        for (const MixedGroupHost& g : m->groups) {
            if (mixed_in_persistent(g)) continue;
            if (g.plan != prev) {
                si = (si + 1) % zlfft_mixed_s::kSideStreams;
                prev = g.plan;
            }
            int rc = mixed_run_group(m, g, m->side[si]);
            if (rc) return rc;
        }
    }
    // the 512-thread class first: its tiles are the longest
    for (int cls = 1; cls >= 0; --cls) {
        for (int pr = 0; pr < 2; ++pr) {
            if (!m->n_items[pr][cls]) continue;
            int* ctr = m->d_counter + 2 * pr + cls;
            ZL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int), st));
            cudaError_t e = pr == 0 ? zlfft::launch_mixed_f32(cls, m->d_mgroups[0], m->d_items[0][cls],
                                                              m->n_items[0][cls], ctr, st, m->num_sms)
                                    : zlfft::launch_mixed_f64(cls, m->d_mgroups[1], m->d_items[1][cls],
                                                              m->n_items[1][cls], ctr, st, m->num_sms);
            if (e != cudaSuccess) return cuda_fail(e, "persistent mixed launch");
            ++m->launches;
        }
    }
    if (big) {
        for (int i = 0; i < zlfft_mixed_s::kSideStreams; ++i) {
            ZL_CUDA(cudaEventRecord(m->ev_join[i], m->side[i]));
            ZL_CUDA(cudaStreamWaitEvent(st, m->ev_join[i], 0));
        }
    }
    return ZLFFT_OK;
}

int mixed_create_impl(zlfft_mixed* out, const zlfft_desc* descs, size_t n, int device) {
    if (!out) return fail(ZLFFT_ERR_INVALID_ARG, "mixed pointer is null");
    *out = nullptr;
    if (n && !descs) return fail(ZLFFT_ERR_INVALID_ARG, "null descriptor array");
    if (n > (size_t)1 << 30) return fail(ZLFFT_ERR_INVALID_ARG, "too many descriptors");
    for (size_t i = 0; i < n; ++i) {
        int rc = mixed_validate(descs[i], i);
        if (rc) return rc;
    }
    if (int rc = mixed_check_overlaps(descs, n)) return rc;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "no CUDA device");
    auto* m = new zlfft_mixed_s();
    m->device = device;
    DeviceGuard dg(device);
    if (cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        mixed_release(m);
        return fail(ZLFFT_ERR_CUDA, "cudaDeviceGetAttribute failed");
    }
    auto dop_of = [](const zlfft_desc& d) {
        if (d.kind == ZLFFT_C2C) return d.op == ZLFFT_FORWARD ? (int)zlfft::kC2CFwd : (int)zlfft::kC2CBwd;
        if (d.op == ZLFFT_FORWARD) return (int)zlfft::kR2CFwd;
        if (d.op == ZLFFT_FORWARD_SQR_MAG) return (int)zlfft::kR2CSqrMag;
        return (int)zlfft::kC2RBwd;
    };
    auto cplx_order = [](const zlfft_desc& d) { return d.kind == ZLFFT_C2C ? d.order : d.order - 1; };
    // sort: complex order descending, then precision, kind, order, op (stable for the data order)
    std::vector<size_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
        const zlfft_desc &a = descs[x], &b = descs[y];
        return std::make_tuple(-cplx_order(a), a.precision, a.kind, a.order, dop_of(a)) <
               std::make_tuple(-cplx_order(b), b.precision, b.kind, b.order, dop_of(b));
    });
    std::map<std::tuple<int, int, int>, zlfft_plan> plan_of;  // (precision, kind, order)
    std::vector<const void*> h_gin(n);
    std::vector<void*> h_gout(n);
    for (size_t j = 0; j < n; ++j) {
        const zlfft_desc& d = descs[idx[j]];
        h_gin[j] = d.in;
        h_gout[j] = d.out;
        const int dop = dop_of(d);
        MixedGroupHost* g = m->groups.empty() ? nullptr : &m->groups.back();
        if (!g || g->prec != d.precision || g->plan->kind != d.kind || g->plan->order != d.order || g->dop != dop) {
            auto key = std::make_tuple(d.precision, d.kind, d.order);
            auto it = plan_of.find(key);
            if (it == plan_of.end()) {
                zlfft_plan p = nullptr;
                // the device's autotuned plan for this size where there is one
                int rc = zlfft_plan_create(&p, d.kind, d.precision, (size_t)d.order, ZLFFT_MODE_TUNED, device);
                if (rc) {
                    mixed_release(m);
                    return rc;
                }
                m->plans.push_back(p);
                if (p->cfft_order > zlfft::kTileMaxP && (rc = ensure_scratch(p)) != ZLFFT_OK) {
                    mixed_release(m);
                    return rc;
                }
                it = plan_of.emplace(key, p).first;
            }
            m->groups.push_back(MixedGroupHost{it->second, d.precision, dop, cplx_order(d), j, 0});
            g = &m->groups.back();
        }
        ++g->count;
    }
    // device block: gather arrays, then per precision the group records and work lists
    std::vector<zlfft::MixedGroup> mg[2];
    std::vector<zlfft::MixedItem> items[2][2];  // [precision][order class]
    std::vector<long long> cost[2][2];
    const size_t gin_off = 0, gout_off = n * sizeof(void*);
    size_t off = 2 * n * sizeof(void*);
    auto align_up = [](size_t v) { return (v + 255) & ~size_t{255}; };
    for (const MixedGroupHost& g : m->groups) {
        if (!mixed_in_persistent(g)) continue;
        const int pr = g.prec == ZLFFT_F32 ? 0 : 1;
        const int cls = zlfft::mixed_class(g.P);
        const int tpc = zlfft::mixed_tpc(g.P);
        const long long tiles = ((long long)g.count + tpc - 1) / tpc;
        for (long long t = 0; t < tiles; ++t) {
            items[pr][cls].push_back(zlfft::MixedItem{(int)mg[pr].size(), (int)t});
            cost[pr][cls].push_back(mixed_tile_cost(g.P));
        }
        mg[pr].push_back(zlfft::MixedGroup{zlfft::TileArgs{}, zlfft::mixed_code(g.dop, g.P)});
    }
    for (int pr = 0; pr < 2; ++pr) {
        for (int cls = 0; cls < 2; ++cls) {
            // longest tiles first (groups are already in descending order; keep it stable)
            std::vector<zlfft::MixedItem>& it = items[pr][cls];
            std::vector<size_t> o(it.size());
            for (size_t i = 0; i < o.size(); ++i) o[i] = i;
            std::stable_sort(o.begin(), o.end(),
                             [&](size_t x, size_t y) { return cost[pr][cls][x] > cost[pr][cls][y]; });
            std::vector<zlfft::MixedItem> sorted(o.size());
            for (size_t i = 0; i < o.size(); ++i) sorted[i] = it[o[i]];
            it.swap(sorted);
            if (it.size() > (size_t)INT32_MAX) {
                mixed_release(m);
                return fail(ZLFFT_ERR_INVALID_ARG, "too many tiles");
            }
            m->n_items[pr][cls] = (int)it.size();
        }
    }
    size_t grp_off[2], item_off[2][2];
    for (int pr = 0; pr < 2; ++pr) {
        off = align_up(off);
        grp_off[pr] = off;
        off += mg[pr].size() * sizeof(zlfft::MixedGroup);
        for (int cls = 0; cls < 2; ++cls) {
            off = align_up(off);
            item_off[pr][cls] = off;
            off += items[pr][cls].size() * sizeof(zlfft::MixedItem);
        }
    }
    // Multi-pass groups: one tensor map per transform for the first pass's bulk
    // copies (the contiguous path's single map cannot describe scattered
    // transforms). A group with any input off 16-byte alignment keeps direct loads.
    std::vector<CUtensorMap> h_maps;
    std::vector<size_t> map_first(m->groups.size(), SIZE_MAX);
    for (MixedGroupHost& g : m->groups) {
        g.in_aligned = true;
        for (size_t i = 0; i < g.count && g.in_aligned; ++i) g.in_aligned = aligned(h_gin[g.first + i], 16);
    }
    for (size_t gi = 0; gi < m->groups.size(); ++gi) {
        const MixedGroupHost& g = m->groups[gi];
        const zlfft_plan_s* gp = g.plan;
        if (mixed_in_persistent(g) || g.P < zlfft::kPassMinP || tile14(gp) || gp->micro >= 0 ||
            g.dop == zlfft::kC2RBwd)
            continue;
        const int* geo = pass_table(gp).first_geom[g.P - zlfft::kPassMinP];
        if (!geo[3]) continue;
        const size_t b = h_maps.size();
        h_maps.resize(b + g.count);
        bool ok = true;
        for (size_t i = 0; i < g.count && ok; ++i)
            ok = zlfft::encode_first_map_one(&h_maps[b + i], h_gin[g.first + i], g.prec == ZLFFT_F64, 1 << g.P,
                                             geo[0], geo[1], geo[2]);
        if (!ok) {
            h_maps.resize(b);
            continue;
        }
        map_first[gi] = b;
    }
    off = align_up(off);
    const size_t maps_off = off;
    off += h_maps.size() * sizeof(CUtensorMap);
    off = align_up(off);
    const size_t counter_off = off;
    off += 4 * sizeof(int);
    if (cudaMalloc(&m->d_mem, off) != cudaSuccess) {
        cudaGetLastError();
        mixed_release(m);
        return fail(ZLFFT_ERR_ALLOC, "mixed batch allocation of %zu bytes failed", off);
    }
    char* base = static_cast<char*>(m->d_mem);
    m->d_gin = reinterpret_cast<const void**>(base + gin_off);
    m->d_gout = reinterpret_cast<void**>(base + gout_off);
    m->d_counter = reinterpret_cast<int*>(base + counter_off);
    for (size_t gi = 0; gi < m->groups.size(); ++gi)
        if (map_first[gi] != SIZE_MAX)
            m->groups[gi].d_maps = base + maps_off + map_first[gi] * sizeof(CUtensorMap);
    // group records now that the gather arrays have device addresses
    {
        size_t k[2] = {0, 0};
        for (const MixedGroupHost& g : m->groups) {
            if (!mixed_in_persistent(g)) continue;
            const int pr = g.prec == ZLFFT_F32 ? 0 : 1;
            mg[pr][k[pr]++].a = mixed_args(m, g);
        }
    }
    cudaError_t e = cudaSuccess;
    if (n) {
        e = cudaMemcpy(base + gin_off, h_gin.data(), n * sizeof(void*), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(base + gout_off, h_gout.data(), n * sizeof(void*), cudaMemcpyHostToDevice);
    }
    for (int pr = 0; pr < 2 && e == cudaSuccess; ++pr) {
        m->d_mgroups[pr] = reinterpret_cast<zlfft::MixedGroup*>(base + grp_off[pr]);
        if (!mg[pr].empty())
            e = cudaMemcpy(m->d_mgroups[pr], mg[pr].data(), mg[pr].size() * sizeof(zlfft::MixedGroup),
                           cudaMemcpyHostToDevice);
        for (int cls = 0; cls < 2 && e == cudaSuccess; ++cls) {
            m->d_items[pr][cls] = reinterpret_cast<zlfft::MixedItem*>(base + item_off[pr][cls]);
            if (!items[pr][cls].empty())
                e = cudaMemcpy(m->d_items[pr][cls], items[pr][cls].data(),
                               items[pr][cls].size() * sizeof(zlfft::MixedItem), cudaMemcpyHostToDevice);
        }
    }
    if (e == cudaSuccess && !h_maps.empty())
        e = cudaMemcpy(base + maps_off, h_maps.data(), h_maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->d_counter, 0, 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->cap_stream, cudaStreamNonBlocking);
    for (int i = 0; i < zlfft_mixed_s::kSideStreams && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&m->side[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ev_join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ev_fork, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        mixed_release(m);
        return cuda_fail(e, "mixed batch set-up");
    }
    *out = m;
    return ZLFFT_OK;
}

// The persistent schedule recorded once into a graph (on the batch's own
// stream, relaxed capture mode), replayed on the caller's stream.
int mixed_graph(zlfft_mixed_s* m, cudaStream_t st) {
    if (!m->graph_exec) {
        const size_t before = m->launches;
        ZL_CUDA(cudaStreamBeginCapture(m->cap_stream, cudaStreamCaptureModeRelaxed));
        int rc = mixed_run(m, ZLFFT_SCHED_PERSISTENT, m->cap_stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(m->cap_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        m->graph = graph;
        ZL_CUDA(cudaGraphInstantiate(&m->graph_exec, m->graph, 0));
        m->graph_launches = m->launches - before;
        m->launches = before;
    }
    ZL_CUDA(cudaGraphLaunch(m->graph_exec, st));
    m->launches += m->graph_launches;
    return ZLFFT_OK;
}
// ------------------------------------------------------------------ the reference's algorithm switch
// get_switch_order<F> of the reference (src/common/zldsp_fft_common_system.hpp:132-157)
// on this host: the same cache queries (sysconf on Linux, with the
// reference's defaults of 32 KiB L1d, 256 KiB L2 and no L3 where a query
// gives nothing) and the same arithmetic.
void host_switch_order(size_t esize, int* max_l1_order, int* switch_order) {
    auto cache = [](int name, long dflt) -> size_t {
        const long v = sysconf(name);
        return (size_t)(v > 0 ? v : dflt);
    };
    auto bit_width = [](size_t x) -> int {
        int w = 0;
        while (x) {
            ++w;
            x >>= 1;
        }
        return w;
    };
    const size_t l1d = cache(_SC_LEVEL1_DCACHE_SIZE, 32768);
    const size_t l2 = cache(_SC_LEVEL2_CACHE_SIZE, 262144);
    const size_t l3 = cache(_SC_LEVEL3_CACHE_SIZE, 0);
    const size_t l1e = l1d / (8 * esize), l2e = l2 / (12 * esize);
    const int l1o = l1e == 0 ? 0 : bit_width(l1e) - 1;
    const int l2o = l2e == 0 ? 0 : bit_width(l2e) - 1;
    int sw = std::max(l1o + 4, l2o);
    if (l3 > (size_t{64} << 20)) {
        const size_t l3e = l3 / (12 * esize);
        sw = std::max(sw, l3e == 0 ? 0 : bit_width(l3e) - 1);
    }
    *max_l1_order = l1o;
    *switch_order = sw;
}

// Unified and per-stage twiddle tables of order `order` (the plan's micro
// order), generated as the plan's own tables are: the bits equal the plan
// table's entries t * 2^(cfft_order - order).
int make_micro_tables(zlfft_plan_s* p, int order) {
    const long long m = 1LL << order;
    const size_t cx_bytes = 2 * p->esize;
    const long long cnt = 3 * m / 4;
    const long long l0 = zlfft::stage_l0(order);
    const long long scnt = m - l0;
    if (cudaMalloc(&p->d_mtw, (size_t)(cnt + 1) * cx_bytes) != cudaSuccess)
        return alloc_fail("micro twiddle", (size_t)(cnt + 1) * cx_bytes);
    if (cudaMalloc(&p->d_mtws, (size_t)(scnt + 1) * cx_bytes) != cudaSuccess)
        return alloc_fail("micro stage twiddle", (size_t)(scnt + 1) * cx_bytes);
    if (p->prec == ZLFFT_F32) {
        twiddle_kernel<float><<<(unsigned)((cnt + 255) / 256), 256, 0, p->stream>>>(static_cast<float2*>(p->d_mtw),
                                                                                     order, cnt);
        stage_table_kernel<float><<<(unsigned)((scnt + 255) / 256), 256, 0, p->stream>>>(
            static_cast<float2*>(p->d_mtws), static_cast<const float2*>(p->d_mtw), order, scnt);
    } else {
        twiddle_kernel<double><<<(unsigned)((cnt + 255) / 256), 256, 0, p->stream>>>(static_cast<double2*>(p->d_mtw),
                                                                                      order, cnt);
        stage_table_kernel<double><<<(unsigned)((scnt + 255) / 256), 256, 0, p->stream>>>(
            static_cast<double2*>(p->d_mtws), static_cast<const double2*>(p->d_mtw), order, scnt);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return cuda_fail(e, "micro twiddle generation");
    return ZLFFT_OK;
}

// Make a plain plan follow the reference's switch (src/common/zldsp_fft_common_init.hpp:305-339):
// a CFFT order at or above switch_order takes the macro path with micro order
// max_l1_order, or max_l1_order - 1 when the difference is odd.
int apply_switch(zlfft_plan_s* p, int max_l1_order, int switch_order) {
    p->max_l1 = max_l1_order;
    p->switch_order = switch_order;
    const int O = p->cfft_order;
    if (O < switch_order) return ZLFFT_OK;  // the micro-only path: the plain plan as it is
    const int m = ((O - max_l1_order) % 2 != 0) ? max_l1_order - 1 : max_l1_order;
    if (m < zlfft::kSegMinM || m > zlfft::kSegMaxM || O - m < 2)
        return fail(ZLFFT_ERR_UNSUPPORTED,
                    "the macro path of CFFT order %d with micro order %d is not built (micro orders %d-%d, at "
                    "least one macro stage)",
                    O, m, zlfft::kSegMinM, zlfft::kSegMaxM);
    DeviceGuard g(p->device);
    int rc = make_micro_tables(p, m);
    if (rc) return rc;
    p->micro = m;
    return ZLFFT_OK;
}

}  // namespace

extern "C" {

int zlfft_plan_create(zlfft_plan* out, int kind, int precision, size_t order, int mode, int device) {
    if (!out) return fail(ZLFFT_ERR_INVALID_ARG, "plan pointer is null");
    *out = nullptr;
    if (kind != ZLFFT_C2C && kind != ZLFFT_R2C) return fail(ZLFFT_ERR_INVALID_ARG, "invalid kind %d", kind);
    if (precision != ZLFFT_F32 && precision != ZLFFT_F64)
        return fail(ZLFFT_ERR_INVALID_ARG, "invalid precision %d", precision);
    if (order > 30) return fail(ZLFFT_ERR_INVALID_ARG, "order %zu out of range", order);
    if (kind == ZLFFT_R2C && order < 1)
        return fail(ZLFFT_ERR_INVALID_ARG, "RFFT order must be >= 1 (the reference underflows at 0)");
    if (mode != ZLFFT_MODE_PLAIN && mode != ZLFFT_MODE_TC_FP16 && mode != ZLFFT_MODE_TUNED && mode != ZLFFT_MODE_FAST &&
        mode != ZLFFT_MODE_HOST)
        return fail(ZLFFT_ERR_UNSUPPORTED, "mode %d not available", mode);
    if (mode == ZLFFT_MODE_TC_FP16 && (kind != ZLFFT_C2C || precision != ZLFFT_F32))
        return fail(ZLFFT_ERR_UNSUPPORTED, "the tensor-core split form is built for CFFT<float>");
    const int cfft_order = kind == ZLFFT_C2C ? (int)order : (int)order - 1;
    if (cfft_order > zlfft::kPassMaxP) return fail(ZLFFT_ERR_UNSUPPORTED, "order %zu above the supported maximum", order);

    auto* p = new zlfft_plan_s();
    p->kind = kind;
    p->prec = precision;
    p->order = (int)order;
    p->cfft_order = cfft_order;
    p->mode = mode;
    p->esize = precision == ZLFFT_F32 ? 4 : 8;
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) {
            delete p;
            return fail(ZLFFT_ERR_CUDA, "no CUDA device");
        }
    }
    p->device = device;
    DeviceGuard g(device);
    if (device >= 0 && device < 64) {
        std::call_once(g_tune_env_once[device], [device]() {
            if (const char* path = getenv("ZLFFT_TUNE_FILE")) tuning_load_impl(device, path, nullptr);
        });
    }
    {
        TuneEntry te;
        if (tune_lookup(device, kind, precision, (int)order, &te)) {
            if (te.chunk_mb > 0) p->chunk_mb = (size_t)te.chunk_mb;
            p->nlanes = te.streams;
            p->use_tma = te.tma;
            p->fuse_split = te.split_fused != 0;
            p->store_tma = te.store_tma;
            if (mode == ZLFFT_MODE_TUNED && te.form == ZLFFT_MODE_TC_FP16) p->tc_form = true;
            if (mode == ZLFFT_MODE_TUNED && te.form == ZLFFT_MODE_FAST) p->fast_form = true;
        }
        if (mode == ZLFFT_MODE_TC_FP16) p->tc_form = true;
        if (mode == ZLFFT_MODE_FAST) p->fast_form = true;
        p->pass_scheme = default_pass_scheme(p);
    }
    cudaError_t e = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        release(p);
        return cuda_fail(e, "cudaDeviceGetAttribute");
    }
    e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->stream2, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        release(p);
        return cuda_fail(e, "cudaStreamCreate");
    }
    (void)tables();
    if (cudaMalloc(&p->d_err, sizeof(int)) != cudaSuccess || cudaMemset(p->d_err, 0, sizeof(int)) != cudaSuccess) {
        release(p);
        return alloc_fail("error-word", sizeof(int));
    }

    const long long m = 1LL << cfft_order;
    p->tw_count = (size_t)(3 * m / 4);
    const size_t cx_bytes = 2 * p->esize;
    e = cudaMalloc(&p->d_tw, (p->tw_count + 1) * cx_bytes);
    if (e != cudaSuccess) {
        release(p);
        return alloc_fail("twiddle", (p->tw_count + 1) * cx_bytes);
    }
    if (p->tw_count > 0) {
        const unsigned blocks = (unsigned)((p->tw_count + 255) / 256);
        if (precision == ZLFFT_F32)
            twiddle_kernel<float><<<blocks, 256, 0, p->stream>>>(static_cast<float2*>(p->d_tw), cfft_order,
                                                                 (long long)p->tw_count);
        else
            twiddle_kernel<double><<<blocks, 256, 0, p->stream>>>(static_cast<double2*>(p->d_tw), cfft_order,
                                                                  (long long)p->tw_count);
    }
    // per-stage tables: N - L0 entries (the stages with sub-length L0 .. N/4)
    {
        const long long l0 = zlfft::stage_l0(cfft_order);
        const long long cnt = m >= 4 * l0 ? m - l0 : 0;
        if (cudaMalloc(&p->d_tws, (size_t)(cnt + 1) * cx_bytes) != cudaSuccess) {
            release(p);
            return alloc_fail("stage twiddle", (size_t)(cnt + 1) * cx_bytes);
        }
        if (cnt > 0) {
            const unsigned blocks = (unsigned)((cnt + 255) / 256);
            if (precision == ZLFFT_F32)
                stage_table_kernel<float><<<blocks, 256, 0, p->stream>>>(
                    static_cast<float2*>(p->d_tws), static_cast<const float2*>(p->d_tw), cfft_order, cnt);
            else
                stage_table_kernel<double><<<blocks, 256, 0, p->stream>>>(
                    static_cast<double2*>(p->d_tws), static_cast<const double2*>(p->d_tw), cfft_order, cnt);
        }
    }
    if (kind == ZLFFT_R2C) {
        const long long cnt = m / 2 + 1;
        if (cudaMalloc(&p->d_rw, cnt * cx_bytes) != cudaSuccess) {
            release(p);
            return alloc_fail("RFFT twiddle", cnt * cx_bytes);
        }
        const unsigned blocks = (unsigned)((cnt + 255) / 256);
        if (precision == ZLFFT_F32)
            rfft_twiddle_kernel<float><<<blocks, 256, 0, p->stream>>>(static_cast<float2*>(p->d_rw), (int)order, cnt);
        else
            rfft_twiddle_kernel<double><<<blocks, 256, 0, p->stream>>>(static_cast<double2*>(p->d_rw), (int)order,
                                                                       cnt);
    }
    if (p->tc_form && cfft_order >= zlfft::kPassMinP) {
        // per-pass tables of the tensor-core passes with L_in > 1: 20 L_in entries each
        size_t total = 0;
        const auto& tt = tables().tc;
        for (int pi = 0; pi < zlfft::kMaxPasses; ++pi) {
            p->tctw_off[pi] = total;
            const int l_in = tt.l_in[cfft_order - zlfft::kPassMinP][pi];
            if (tt.fn[cfft_order - zlfft::kPassMinP][pi][0] && l_in > 1) total += 20 * (size_t)l_in;
        }
        if (total) {
            if (cudaMalloc(&p->d_tctw, total * cx_bytes) != cudaSuccess) {
                release(p);
                return alloc_fail("tensor-core twiddle", total * cx_bytes);
            }
            for (int pi = 0; pi < zlfft::kMaxPasses; ++pi) {
                const int l_in = tt.l_in[cfft_order - zlfft::kPassMinP][pi];
                if (!tt.fn[cfft_order - zlfft::kPassMinP][pi][0] || l_in <= 1) continue;
                const int cnt = 20 * l_in;
                tc_pass_table_kernel<<<(cnt + 255) / 256, 256, 0, p->stream>>>(
                    static_cast<float2*>(p->d_tctw) + p->tctw_off[pi], static_cast<const float2*>(p->d_tw), (int)m,
                    l_in);
            }
        }
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) {
        release(p);
        return cuda_fail(e, "twiddle generation");
    }
    if (mode == ZLFFT_MODE_HOST) {
        int l1o = 0, swo = 0;
        host_switch_order(p->esize, &l1o, &swo);
        const int rc = apply_switch(p, l1o, swo);
        if (rc) {
            release(p);
            return rc;
        }
    }
    *out = p;
    return ZLFFT_OK;
}

int zlfft_plan_create_hybrid(zlfft_plan* out, int kind, int precision, size_t order, int max_l1_order,
                             int switch_order, int device) {
    if (!out) return fail(ZLFFT_ERR_INVALID_ARG, "plan pointer is null");
    *out = nullptr;
    if (max_l1_order < 0 || max_l1_order > 30 || switch_order < 0)
        return fail(ZLFFT_ERR_INVALID_ARG, "invalid switch (max_l1_order %d, switch_order %d)", max_l1_order,
                    switch_order);
    zlfft_plan p = nullptr;
    int rc = zlfft_plan_create(&p, kind, precision, order, ZLFFT_MODE_PLAIN, device);
    if (rc) return rc;
    rc = apply_switch(p, max_l1_order, switch_order);
    if (rc) {
        release(p);
        return rc;
    }
    *out = p;
    return ZLFFT_OK;
}

int zlfft_host_switch_order(int precision, size_t* max_l1_order, size_t* switch_order) {
    if (!max_l1_order || !switch_order) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    if (precision != ZLFFT_F32 && precision != ZLFFT_F64)
        return fail(ZLFFT_ERR_INVALID_ARG, "invalid precision %d", precision);
    int l1o = 0, swo = 0;
    host_switch_order(precision == ZLFFT_F32 ? 4 : 8, &l1o, &swo);
    *max_l1_order = (size_t)l1o;
    *switch_order = (size_t)swo;
    return ZLFFT_OK;
}

int zlfft_plan_get_micro_order(zlfft_plan plan, int* micro_order) {
    if (!plan || !micro_order) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    *micro_order = plan->micro;
    return ZLFFT_OK;
}

int zlfft_plan_destroy(zlfft_plan plan) {
    release(plan);
    return ZLFFT_OK;
}

int zlfft_plan_get_size(zlfft_plan plan, size_t* size) {
    if (!plan || !size) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    *size = size_t{1} << plan->order;
    return ZLFFT_OK;
}

int zlfft_plan_get_order(zlfft_plan plan, size_t* order) {
    if (!plan || !order) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    *order = (size_t)plan->order;
    return ZLFFT_OK;
}

int zlfft_exec_host(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                    void* out0, void* out1) {
    if (!plan) return fail(ZLFFT_ERR_INVALID_ARG, "null plan");
    return exec_host_impl(plan, op, in_layout, out_layout, in0, in1, out0, out1, 1);
}

int zlfft_exec_host_batched(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0,
                            const void* in1, void* out0, void* out1, size_t batch) {
    if (!plan) return fail(ZLFFT_ERR_INVALID_ARG, "null plan");
    return exec_host_impl(plan, op, in_layout, out_layout, in0, in1, out0, out1, batch);
}

int zlfft_exec_device(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                      void* out0, void* out1, size_t batch, size_t in_stride, size_t out_stride, void* stream) {
    if (!plan) return fail(ZLFFT_ERR_INVALID_ARG, "null plan");
    return exec_device_impl(plan, op, in_layout, out_layout, in0, in1, out0, out1, batch, in_stride, out_stride,
                            static_cast<cudaStream_t>(stream));
}

int zlfft_stft_device(zlfft_plan plan, int op, int out_layout, const void* signal, size_t hop, const void* window,
                      void* out0, void* out1, size_t n_frames, size_t out_stride, void* stream) {
    if (!plan) return fail(ZLFFT_ERR_INVALID_ARG, "null plan");
    return stft_impl(plan, op, out_layout, signal, hop, window, out0, out1, n_frames, out_stride,
                     static_cast<cudaStream_t>(stream));
}

int zlfft_istft_device(zlfft_plan plan, int in_layout, const void* in0, const void* in1, size_t in_stride,
                       const void* filter, const void* window, size_t hop, size_t n_frames, void* signal, void* stream) {
    if (!plan) return fail(ZLFFT_ERR_INVALID_ARG, "null plan");
    return istft_impl(plan, in_layout, in0, in1, in_stride, filter, window, hop, n_frames, signal,
                      static_cast<cudaStream_t>(stream));
}

int zlfft_exec_device_noalloc(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0,
                              const void* in1, void* out0, void* out1, size_t batch, size_t in_stride,
                              size_t out_stride, void* stream) {
    if (!plan) return fail(ZLFFT_ERR_INVALID_ARG, "null plan");
    return exec_device_noalloc_impl(plan, op, in_layout, out_layout, in0, in1, out0, out1, batch, in_stride,
                                    out_stride, static_cast<cudaStream_t>(stream));
}

int zlfft_plan_take_launch_count(zlfft_plan plan, size_t* launches) {
    if (!plan || !launches) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    *launches = plan->launches.exchange(0);
    return ZLFFT_OK;
}

int zlfft_plan_copy_twiddles(zlfft_plan plan, void* host_out, size_t capacity_elems, size_t* count) {
    if (!plan || !count) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    *count = plan->tw_count;
    if (!host_out) return ZLFFT_OK;
    if (capacity_elems < plan->tw_count) return fail(ZLFFT_ERR_INVALID_ARG, "capacity too small");
    DeviceGuard g(plan->device);
    ZL_CUDA(cudaMemcpy(host_out, plan->d_tw, plan->tw_count * 2 * plan->esize, cudaMemcpyDeviceToHost));
    return ZLFFT_OK;
}

int zlfft_plan_device_status(zlfft_plan plan, int* status) {
    if (!plan || !status) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    DeviceGuard g(plan->device);
    ZL_CUDA(cudaDeviceSynchronize());
    ZL_CUDA(cudaMemcpy(status, plan->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    ZL_CUDA(cudaMemset(plan->d_err, 0, sizeof(int)));
    return *status ? ZLFFT_ERR_DEVICE_TIMEOUT : ZLFFT_OK;
}

int zlfft_selftest_bounded_wait(int device, int* status) {
    if (!status) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    DeviceGuard g(device);
    int* d = nullptr;
    ZL_CUDA(cudaMalloc(&d, sizeof(int)));
    cudaMemset(d, 0, sizeof(int));
    selftest_wait_kernel<<<1, 64>>>(d, 4096u);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "selftest");
    return ZLFFT_OK;
}

int zlfft_mixed_create(zlfft_mixed* mixed, const zlfft_desc* descs, size_t n, int device) {
    return mixed_create_impl(mixed, descs, n, device);
}

int zlfft_mixed_exec(zlfft_mixed mixed, int schedule, void* stream) {
    if (!mixed) return fail(ZLFFT_ERR_INVALID_ARG, "null mixed batch");
    if (schedule < ZLFFT_SCHED_PER_ORDER || schedule > ZLFFT_SCHED_GRAPH)
        return fail(ZLFFT_ERR_INVALID_ARG, "invalid schedule %d", schedule);
    std::lock_guard<std::mutex> lock(mixed->mu);
    DeviceGuard g(mixed->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (schedule == ZLFFT_SCHED_GRAPH) return mixed_graph(mixed, st);
    return mixed_run(mixed, schedule, st);
}

int zlfft_mixed_take_launch_count(zlfft_mixed mixed, size_t* launches) {
    if (!mixed || !launches) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lock(mixed->mu);
    *launches = mixed->launches.exchange(0);
    return ZLFFT_OK;
}

int zlfft_mixed_device_status(zlfft_mixed mixed, int* status) {
    if (!mixed || !status) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    int any = 0;
    for (zlfft_plan p : mixed->plans) {
        int s = 0;
        int rc = zlfft_plan_device_status(p, &s);
        if (rc && rc != ZLFFT_ERR_DEVICE_TIMEOUT) return rc;
        any |= s;
    }
    *status = any;
    return any ? ZLFFT_ERR_DEVICE_TIMEOUT : ZLFFT_OK;
}

int zlfft_mixed_destroy(zlfft_mixed mixed) {
    mixed_release(mixed);
    return ZLFFT_OK;
}

int zlfft_exec_mixed_device(const zlfft_desc* descs, size_t n, void* stream) {
    zlfft_mixed m = nullptr;
    int rc = mixed_create_impl(&m, descs, n, -1);
    if (rc) return rc;
    {
        DeviceGuard g(m->device);
        rc = mixed_run(m, ZLFFT_SCHED_PERSISTENT, static_cast<cudaStream_t>(stream));
        const cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamSynchronize");
    }
    mixed_release(m);
    return rc;
}

int zlfft_selftest_tc_dft16(int device, const float* host_in, float* host_out, int* status) {
    if (!host_in || !host_out || !status) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    DeviceGuard g(device);
    const size_t bytes = 128 * 16 * sizeof(float2);
    float2 tw[16];
    for (int t = 0; t < 16; ++t) {
        const double a = -2.0 * 3.141592653589793 * t / 16.0;
        tw[t] = make_float2((float)cos(a), (float)sin(a));
    }
    void* d = nullptr;
    ZL_CUDA(cudaMalloc(&d, 2 * bytes + sizeof(tw) + 256));
    char* base = static_cast<char*>(d);
    float2* din = reinterpret_cast<float2*>(base);
    float2* dout = reinterpret_cast<float2*>(base + bytes);
    float2* dtw = reinterpret_cast<float2*>(base + 2 * bytes);
    int* derr = reinterpret_cast<int*>(base + 2 * bytes + sizeof(tw));
    cudaError_t e = cudaMemcpy(din, host_in, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dtw, tw, sizeof(tw), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(dout, 0, bytes);
    if (e == cudaSuccess) e = zlfft::tc_selftest_launch(din, dout, dtw, derr, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(host_out, dout, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(status, derr, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "tensor-core self-test");
    return ZLFFT_OK;
}

const char* zlfft_last_error(void) { return g_last_error.c_str(); }

const char* zlfft_version(void) { return "zlfft-b200 0.1 (sm_100a)"; }

}  // extern "C"

namespace {

// One candidate plan timed on `batch` transforms: forward AoS -> AoS.
int time_candidate(int device, int kind, int prec, int order, const TuneEntry& c, const void* in, void* out,
                   size_t batch, cudaStream_t st, double* ms) {
    zlfft_plan p = nullptr;
    int rc = zlfft_plan_create(&p, kind, prec, (size_t)order, c.form, device);
    if (rc) return rc;
    p->chunk_mb = c.chunk_mb > 0 ? (size_t)c.chunk_mb : p->chunk_mb;
    p->nlanes = c.streams;
    p->use_tma = c.tma;
    p->fuse_split = c.split_fused != 0;
    p->store_tma = c.store_tma;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    constexpr int kReps = 5;
    for (int i = 0; i < 2 && !rc; ++i)
        rc = exec_device_impl(p, ZLFFT_FORWARD, ZLFFT_AOS, ZLFFT_AOS, in, nullptr, out, nullptr, batch, 0, 0, st);
    if (!rc) {
        cudaEventRecord(e0, st);
        for (int i = 0; i < kReps && !rc; ++i)
            rc = exec_device_impl(p, ZLFFT_FORWARD, ZLFFT_AOS, ZLFFT_AOS, in, nullptr, out, nullptr, batch, 0, 0, st);
        cudaEventRecord(e1, st);
    }
    cudaError_t e = cudaStreamSynchronize(st);
    float t = 0;
    if (!rc && e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int st_err = 0;
    cudaMemcpy(&st_err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    release(p);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "autotune timing");
    if (st_err) return fail(ZLFFT_ERR_DEVICE_TIMEOUT, "a device-side wait ran out during autotuning");
    *ms = t / kReps;
    return ZLFFT_OK;
}

int autotune_impl(int device, int kind, int prec, size_t lo, size_t hi) {
    if (kind != ZLFFT_C2C && kind != ZLFFT_R2C) return fail(ZLFFT_ERR_INVALID_ARG, "invalid kind %d", kind);
    if (prec != ZLFFT_F32 && prec != ZLFFT_F64) return fail(ZLFFT_ERR_INVALID_ARG, "invalid precision %d", prec);
    const size_t min_order = kind == ZLFFT_R2C ? 1 : 0;
    const size_t max_order = (size_t)zlfft::kPassMaxP + (kind == ZLFFT_R2C ? 1 : 0);
    if (lo < min_order || hi > max_order || lo > hi)
        return fail(ZLFFT_ERR_UNSUPPORTED, "orders %zu..%zu outside %zu..%zu", lo, hi, min_order, max_order);
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "no CUDA device");
    DeviceGuard g(device);
    const size_t es = prec == ZLFFT_F32 ? 4 : 8;
    const size_t budget = size_t{512} << 20;
    const size_t n_hi = size_t{1} << hi;
    const size_t one = 2 * es * (n_hi + 2);  // largest single transform, either side
    const size_t bytes = std::max(budget, one) + 256;
    void* d_in = nullptr;
    void* d_out = nullptr;
    if (cudaMalloc(&d_in, bytes) != cudaSuccess || cudaMalloc(&d_out, bytes) != cudaSuccess) {
        cudaGetLastError();
        if (d_in) cudaFree(d_in);
        return fail(ZLFFT_ERR_ALLOC, "autotune buffers of %zu bytes failed", bytes);
    }
    cudaStream_t st = nullptr;
    int rc = ZLFFT_OK;
    cudaError_t e = cudaMemset(d_in, 0x3c, bytes);  // every float about 0.0115
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = cuda_fail(e, "autotune set-up");
    for (size_t order = lo; order <= hi && !rc; ++order) {
        const size_t n = size_t{1} << order;
        const int cfft_order = kind == ZLFFT_C2C ? (int)order : (int)order - 1;
        const size_t per_in = kind == ZLFFT_C2C ? 2 * es * n : es * n;
        const size_t per_out = kind == ZLFFT_C2C ? 2 * es * n : 2 * es * (n / 2 + 1);
        const size_t batch = std::max<size_t>(1, budget / std::max(per_in, per_out));
        std::vector<TuneEntry> cands;
        const bool tc_ok = kind == ZLFFT_C2C && prec == ZLFFT_F32 && cfft_order >= zlfft::kPassMinP;
        if (cfft_order >= zlfft::kPassMinP) {
            for (int form : {ZLFFT_MODE_PLAIN, ZLFFT_MODE_FAST, ZLFFT_MODE_TC_FP16}) {
                if (form == ZLFFT_MODE_TC_FP16 && !tc_ok) continue;
                for (int chunk : {16, 32, 48, 96, 192})
                    for (int streams : {1, 2})
                        for (int tma : {0, 1})
                            for (int fused : {0, 1})
                                for (int store : {0, 1}) {
                                    if (fused && kind != ZLFFT_R2C) continue;
                                    TuneEntry c;
                                    c.chunk_mb = chunk;
                                    c.streams = streams;
                                    c.tma = tma;
                                    c.form = form;
                                    c.split_fused = fused;
                                    c.store_tma = store;
                                    cands.push_back(c);
                                }
            }
        } else {
            for (int form : {ZLFFT_MODE_PLAIN, ZLFFT_MODE_FAST}) {
                if (form == ZLFFT_MODE_FAST && cfft_order < 11) continue;  // no middle radix-16 group
                for (int tma : {1, 0}) {
                    TuneEntry c;
                    c.chunk_mb = 0;
                    c.streams = 1;
                    c.tma = tma;
                    c.form = form;
                    cands.push_back(c);
                }
            }
        }
        TuneEntry best;
        double best_gbs = -1, def_gbs = 0;
        for (const TuneEntry& c : cands) {
            double ms = 0;
            rc = time_candidate(device, kind, prec, (int)order, c, d_in, d_out, batch, st, &ms);
            if (rc) break;
            const double gbs = (double)batch * (double)(per_in + per_out) / (ms * 1e6);
            const int store_default = prec == ZLFFT_F32 ? 1 : 0;
            const bool is_default = c.form == ZLFFT_MODE_PLAIN && c.tma == 1 && c.split_fused == 0 &&
                                    (c.chunk_mb == 0 || (c.chunk_mb == 48 && c.streams == 2 &&
                                                         c.store_tma == store_default));
            if (is_default) def_gbs = gbs;
            if (gbs > best_gbs) {
                best_gbs = gbs;
                best = c;
            }
        }
        if (rc) break;
        best.gbs = best_gbs;
        best.gbs_default = def_gbs;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[std::make_tuple(device, kind, prec, (int)order)] = best;
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(d_in);
    cudaFree(d_out);
    return rc;
}

}  // namespace

extern "C" {

int zlfft_autotune(int device, int kind, int precision, size_t order_lo, size_t order_hi) {
    return autotune_impl(device, kind, precision, order_lo, order_hi);
}

int zlfft_tuning_get(int device, int kind, int precision, size_t order, zlfft_tuning* out) {
    if (!out) return fail(ZLFFT_ERR_INVALID_ARG, "null argument");
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "no CUDA device");
    TuneEntry e;
    if (order > 64 || !tune_lookup(device, kind, precision, (int)order, &e))
        return fail(ZLFFT_ERR_UNSUPPORTED, "no tuning entry for this size");
    out->chunk_mb = e.chunk_mb;
    out->streams = e.streams;
    out->tma = e.tma;
    out->form = e.form;
    out->split_fused = e.split_fused;
    out->store_tma = e.store_tma;
    out->gbs = e.gbs;
    out->gbs_default = e.gbs_default;
    return ZLFFT_OK;
}

int zlfft_tuning_save(int device, const char* path) {
    if (!path) return fail(ZLFFT_ERR_INVALID_ARG, "null path");
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "no CUDA device");
    std::string name;
    int sms = 0;
    int rc = gpu_identity(device, &name, &sms);
    if (rc) return rc;
    FILE* f = fopen(path, "w");
    if (!f) return fail(ZLFFT_ERR_INVALID_ARG, "cannot write tuning file %s", path);
    fprintf(f, "# zlfft tuning table: entry kind precision order chunk_mb streams tma form split_fused store_tma "
               "gbs gbs_default\n");
    fprintf(f, "gpu %s sms %d\n", name.c_str(), sms);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (const auto& kv : g_tune) {
            if (std::get<0>(kv.first) != device) continue;
            const TuneEntry& e = kv.second;
            fprintf(f, "entry %d %d %d %d %d %d %d %d %d %.1f %.1f\n", std::get<1>(kv.first), std::get<2>(kv.first),
                    std::get<3>(kv.first), e.chunk_mb, e.streams, e.tma, e.form, e.split_fused, e.store_tma, e.gbs,
                    e.gbs_default);
        }
    }
    if (fclose(f) != 0) return fail(ZLFFT_ERR_INVALID_ARG, "writing %s failed", path);
    return ZLFFT_OK;
}

int zlfft_tuning_load(int device, const char* path, size_t* loaded) {
    if (!path) return fail(ZLFFT_ERR_INVALID_ARG, "null path");
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(ZLFFT_ERR_CUDA, "no CUDA device");
    return tuning_load_impl(device, path, loaded);
}

int zlfft_tuning_clear(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.clear();
    return ZLFFT_OK;
}

}  // extern "C"
