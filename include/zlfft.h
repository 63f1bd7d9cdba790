/* libzlfft_cuda — C ABI of the B200 FFT engine that stands in for
 * zldsp::fft::CFFT<F> and zldsp::fft::RFFT<F> (ZL-Audio/zldsp_fft).
 *
 * The reference is a header-only C++ library; its "binding surface" is the
 * two class templates. Every entry point below names the reference member it
 * replaces (file:line within the reference project). The C++ drop-in headers
 * in include/zldsp_fft_cuda/ implement those classes over this ABI.
 *
 * Conventions (identical to the reference):
 *   forward   X[k] = sum_n x[n] exp(-2 pi i k n / N)
 *   backward  unnormalised inverse: CFFT backward(forward(x)) = N * x,
 *             RFFT backward(forward(x)) = (N/2) * x
 *   RFFT forward writes N/2+1 bins (DC and Nyquist with zero imaginary part);
 *   forward_sqr_mag writes the N/2+1 values re^2 + im^2.
 *
 * All functions return ZLFFT_OK (0) or a negative status; the message of the
 * calling thread's last failure is returned by zlfft_last_error().
 */
#ifndef ZLFFT_H_
#define ZLFFT_H_

#include <stddef.h>

#if defined(__GNUC__)
#define ZLFFT_API __attribute__((visibility("default")))
#else
#define ZLFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zlfft_plan_s* zlfft_plan;

/* status codes */
#define ZLFFT_OK 0
#define ZLFFT_ERR_INVALID_ARG (-1)
#define ZLFFT_ERR_UNSUPPORTED (-2)
#define ZLFFT_ERR_ALIGNMENT (-3)
#define ZLFFT_ERR_CUDA (-4)
#define ZLFFT_ERR_ALLOC (-5)
#define ZLFFT_ERR_DEVICE_TIMEOUT (-6)

/* transform kind */
#define ZLFFT_C2C 0 /* CFFT<F> */
#define ZLFFT_R2C 1 /* RFFT<F> */

/* precision */
#define ZLFFT_F32 0
#define ZLFFT_F64 1

/* complex layout: AoS = interleaved std::complex<F>[], SoA = split {F* re, F* im} */
#define ZLFFT_AOS 0
#define ZLFFT_SOA 1

/* operation */
#define ZLFFT_FORWARD 0
#define ZLFFT_BACKWARD 1
#define ZLFFT_FORWARD_SQR_MAG 2 /* RFFT only */

/* computation form */
#define ZLFFT_MODE_PLAIN 0   /* reference's Stockham radix-4/8 DIT on CUDA cores */
#define ZLFFT_MODE_TC_FP16 1 /* radix-16 sub-DFTs on tensor cores, split hi/lo FP16 */
/* (2 and 3 are not used) */
#define ZLFFT_MODE_TUNED 4   /* the autotuned plan of this device and size (see zlfft_autotune) */
#define ZLFFT_MODE_FAST 5    /* plain CUDA-core form whose multi-pass radix-16 groups build their
                                twiddles from two table values (fewer loads): within the FP bar,
                                not bit-identical to the reference; single-tile sizes as PLAIN */
#define ZLFFT_MODE_HOST 6    /* PLAIN, following the reference's own algorithm switch as the caches of
                                THIS host set it (see zlfft_host_switch_order): bit-identical (FP32)
                                to the reference's output on this host, macro path included */

/* Create a plan for one transform size.
 * Replaces the constructors CFFT<F>::CFFT(size_t order)
 * (src/zldsp_fft_cfft.hpp:19-23) and RFFT<F>::RFFT(size_t order)
 * (src/zldsp_fft_rfft.hpp:24-53). order is log2 of the transform length N
 * (RFFT: real length): CFFT orders 0-26, RFFT orders 1-27 (ZLFFT_ERR_UNSUPPORTED
 * above). Twiddle tables are generated on the device in FP64 and rounded to
 * the plan's precision. device < 0 means the current device. */
ZLFFT_API int zlfft_plan_create(zlfft_plan* plan, int kind, int precision, size_t order, int mode, int device);

/* As zlfft_plan_create with mode ZLFFT_MODE_PLAIN, following the reference's
 * algorithm switch with the given values instead of the arithmetic of one
 * path for every order (src/common/zldsp_fft_common_init.hpp:305-339, the
 * constructors' init_cfft_state): a CFFT whose order is >= switch_order (for
 * an RFFT, its inner CFFT of order - 1) runs the reference's macro path -
 * radix-4 Cooley-Tukey DIF stages (src/common/zldsp_fft_common_radix.hpp:670-843),
 * then a Stockham FFT of the micro order per segment and a digit-reversed
 * transposed store (src/common/zldsp_fft_common_execute.hpp:174-272) - with
 * micro order max_l1_order, or max_l1_order - 1 when order - max_l1_order is
 * odd. Below switch_order the plan is the plain micro-only plan. With the
 * (max_l1_order, switch_order) that get_switch_order<F>()
 * (src/common/zldsp_fft_common_system.hpp:132-157) returns on some host, the
 * FP32 output is bit-identical to the reference's on that host (FP64: within
 * the FP64 bar). Micro orders 8-12 are built (ZLFFT_ERR_UNSUPPORTED
 * otherwise). Macro-path plans run through zlfft_exec_host*, zlfft_exec_device
 * and zlfft_exec_device_noalloc; the STFT entry points refuse them. */
ZLFFT_API int zlfft_plan_create_hybrid(zlfft_plan* plan, int kind, int precision, size_t order, int max_l1_order,
                                       int switch_order, int device);

/* The (max_l1_order, switch_order) the reference computes on this host for
 * precision F (get_switch_order<F>, src/common/zldsp_fft_common_system.hpp:132-157):
 * the same cache-size queries (sysconf on Linux, the reference's defaults
 * where a query gives nothing) and arithmetic. ZLFFT_MODE_HOST plans use them. */
ZLFFT_API int zlfft_host_switch_order(int precision, size_t* max_l1_order, size_t* switch_order);

/* The micro order of a plan on the macro path, or -1 when it runs the
 * micro-only path. No reference counterpart (CFFTState::micro_cfft_order,
 * src/common/zldsp_fft_common_init.hpp:25-43, is internal there). */
ZLFFT_API int zlfft_plan_get_micro_order(zlfft_plan plan, int* micro_order);

/* Release a plan and every buffer it owns. Replaces the reference objects'
 * destructors (members freed by hwy::AlignedFreeUniquePtr,
 * src/common/zldsp_fft_common_init.hpp:28-42). */
ZLFFT_API int zlfft_plan_destroy(zlfft_plan plan);

/* N = 2^order. Replaces CFFT::get_size (src/zldsp_fft_cfft.hpp:25-27) and
 * RFFT::get_size (src/zldsp_fft_rfft.hpp:55-57). */
ZLFFT_API int zlfft_plan_get_size(zlfft_plan plan, size_t* size);

/* Replaces CFFT::get_order (src/zldsp_fft_cfft.hpp:29-31) and
 * RFFT::get_order (src/zldsp_fft_rfft.hpp:59-61). */
ZLFFT_API int zlfft_plan_get_order(zlfft_plan plan, size_t* order);

/* One transform on HOST buffers, synchronous (the output is valid on return),
 * exactly as the reference's member functions behave:
 *   CFFT forward/backward, 8 overloads (src/zldsp_fft_cfft.hpp:38-103):
 *     op = FORWARD|BACKWARD, in_layout/out_layout = AOS|SOA;
 *     AoS uses in0/out0 (complex array), SoA uses (in0 = re, in1 = im).
 *   RFFT::forward(F*, C*) / forward(F*, std::array<F*,2>) (src/zldsp_fft_rfft.hpp:68-80):
 *     op = FORWARD, in0 = real input, out_layout selects AoS/SoA bins.
 *   RFFT::backward(C*, F*) / backward(std::array<F*,2>, F*) (src/zldsp_fft_rfft.hpp:86-98):
 *     op = BACKWARD, in_layout selects AoS/SoA bins, out0 = real output.
 *   RFFT::forward_sqr_mag(F*, F*) (src/zldsp_fft_rfft.hpp:104-109):
 *     op = FORWARD_SQR_MAG, in0 = real input, out0 = N/2+1 reals.
 * Inputs are not modified. CFFT may run in place (in == out, same layout). */
ZLFFT_API int zlfft_exec_host(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                    void* out0, void* out1);

/* As zlfft_exec_host for `batch` transforms laid out back to back (stride =
 * the transform's own element count). No reference counterpart: a batched
 * form of the calls above, staged through the plan's pinned buffers. */
ZLFFT_API int zlfft_exec_host_batched(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0,
                            const void* in1, void* out0, void* out1, size_t batch);

/* Batched transforms on DEVICE buffers, asynchronous on `stream`
 * (a cudaStream_t; NULL = legacy default stream). No reference counterpart:
 * the device-pointer batched entry point that sits beside the reference's
 * calls above. Transform b reads element e at in + b*in_stride + e and writes
 * out + b*out_stride + e, strides counted in elements of the buffer's own
 * type (complex for complex buffers, real for real buffers; 0 = dense).
 * Pointers must be aligned to the element type (8 B f32 complex, 16 B f64
 * complex); RFFT real buffers need an even stride. In place: an output may
 * share memory with an input only from the same start with the same byte
 * stride (CFFT with equal strides; RFFT with real stride 2*(N/2+1), the
 * padded layout); other overlaps with batch > 1 are refused
 * (ZLFFT_ERR_INVALID_ARG). The multi-pass sizes
 * (complex order >= 14) pass their intermediates through the plan's scratch,
 * so calls on one plan must not overlap on the device: issue them on one
 * stream, order the streams with events, or give each stream its own plan. */
ZLFFT_API int zlfft_exec_device(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0, const void* in1,
                      void* out0, void* out1, size_t batch, size_t in_stride, size_t out_stride, void* stream);

/* Short-time Fourier transform front end on DEVICE buffers: frame f of a
 * real signal is signal[f*hop + n] * window[n], n < N (N = the RFFT plan's
 * real length), and each frame goes through RFFT::forward (op FORWARD, bins
 * in out_layout AoS or SoA) or RFFT::forward_sqr_mag (op FORWARD_SQR_MAG,
 * N/2+1 reals) (src/zldsp_fft_rfft.hpp:68-80, :104-109), frame f's output at
 * out + f*out_stride (0 = dense). One launch: frames are read straight from the
 * signal and windowed as they are loaded; no framed copy is made. window NULL
 * means a rectangular window. hop must be even; the signal must hold
 * (n_frames - 1) * hop + N samples. Frame orders up to 15 in FP32 (N <= 32768), 14 in FP64. No
 * reference counterpart: a spectrum analyser built on the reference calls
 * forward_sqr_mag frame by frame on copies it windows itself. */
ZLFFT_API int zlfft_stft_device(zlfft_plan plan, int op, int out_layout, const void* signal, size_t hop,
                                const void* window, void* out0, void* out1, size_t n_frames, size_t out_stride,
                                void* stream);

/* Inverse STFT with overlap-add on DEVICE buffers, the backward-side fusion of
 * the STFT: frame f's bins (N/2+1 complex, AoS in0 or SoA in0/in1, frame f at
 * + f*in_stride, 0 = dense) are multiplied by filter[k] (N/2+1 complex;
 * NULL = none; each complex product rounded operation by operation), go
 * through RFFT::backward (src/zldsp_fft_rfft.hpp:86-100; unnormalised), are
 * multiplied by window[n] (N reals; NULL = none) and added into
 * signal[f*hop + n]. The signal ((n_frames - 1) * hop + N reals) is written,
 * not accumulated into: each real is the sum of its frames' terms in
 * ascending frame order starting from zero, one rounding per term, so the
 * result is that of a sequential loop over frames, bit for bit. hop must be
 * even and divide N. Frame orders 10-14 (FP32) or 10-13 (FP64). With the
 * bins of a zero-padded signal and a filter's spectrum this is overlap-add
 * fast convolution. No reference counterpart: the reference offers the
 * per-frame RFFT::backward only. */
ZLFFT_API int zlfft_istft_device(zlfft_plan plan, int in_layout, const void* in0, const void* in1, size_t in_stride,
                                 const void* filter, const void* window, size_t hop, size_t n_frames, void* signal,
                                 void* stream);

/* As zlfft_exec_device, for callers that cannot allocate device memory when
 * they run a transform: a real-time audio thread (an allocation can block
 * for an unbounded time, and a missed deadline is an audible glitch), or a
 * host whose device memory is all handed to its own pool. No reference
 * counterpart: the reference allocates everything in its constructors.
 *
 * Multi-pass orders (complex order 14 and up, except the FP32 CFFT of order
 * 14 and the FP32 RFFT of order 15, which run one tile per transform) and
 * plans on the reference's macro path pass their intermediates through a
 * scratch array built into the library (64 MiB of device memory, reserved on
 * every GPU that loads the library and held until the process exits), instead
 * of the plan's scratch that zlfft_exec_device allocates on first use. This
 * call allocates nothing and creates no streams or events; the other sizes
 * need no scratch and run exactly as in zlfft_exec_device. Results are
 * identical to zlfft_exec_device's.
 *  - Limit: one transform must fit one 32 MiB half of the array: CFFT order
 *    <= 22 (FP32) / 21 (FP64), RFFT order <= 23 (FP32) / 22 (FP64); larger
 *    orders are rejected with ZLFFT_ERR_UNSUPPORTED.
 *  - The first call on each device that needs the array looks up its device
 *    address (cudaGetSymbolAddress), which may make the driver load the
 *    library's device code; make that first call during set-up, before any
 *    real-time section. A failed lookup is reported and retried next call.
 *  - Every call shares the one array and leaves its contents behind (nothing
 *    in it needs to start at zero). Calls whose work overlaps on the GPU
 *    (different streams, or different plans at once) race on it: serialise
 *    them, e.g. on one stream. */
ZLFFT_API int zlfft_exec_device_noalloc(zlfft_plan plan, int op, int in_layout, int out_layout, const void* in0,
                                        const void* in1, void* out0, void* out1, size_t batch, size_t in_stride,
                                        size_t out_stride, void* stream);

/* Number of CUDA kernels this plan has launched since the previous call
 * (diagnostics for benchmarks). */
ZLFFT_API int zlfft_plan_take_launch_count(zlfft_plan plan, size_t* launches);

/* Copy the plan's unified twiddle table T[t] = exp(-2 pi i t / M), t < 3M/4,
 * to host memory (M = CFFT length; RFFT plans: N/2), as interleaved
 * re/im pairs of the plan precision. `count` receives 3M/4. Diagnostics: lets
 * a caller compare the device-generated table with the reference's. */
ZLFFT_API int zlfft_plan_copy_twiddles(zlfft_plan plan, void* host_out, size_t capacity_elems, size_t* count);

/* Synchronise the plan's device, then read and clear the plan's device error
 * word. Kernels bound every wait they perform (on a TMA completion barrier or
 * on another CTA's progress); a wait that runs out of its iteration limit
 * sets a bit here and the kernel returns early instead of hanging the GPU.
 * Returns ZLFFT_ERR_DEVICE_TIMEOUT if *status != 0. No reference counterpart
 * (the reference runs on one CPU thread and never waits). */
ZLFFT_API int zlfft_plan_device_status(zlfft_plan plan, int* status);

/* Failure-detection self-test: runs one kernel that waits on a barrier that
 * never completes, with a short poll limit, and returns in *status the error
 * word the kernel left (kDevErrWaitTimeout = 1 when the bounded wait gave up
 * as designed). The GPU context stays usable. No reference counterpart. */
ZLFFT_API int zlfft_selftest_bounded_wait(int device, int* status);

/* Tensor-core self-test: 128 independent 16-point forward DFTs of
 * host_in (128 x 16 interleaved complex FP32) computed by one CTA with
 * tcgen05 MMAs on split FP16 hi/lo operands accumulated in FP32 (the
 * building block of the ZLFFT_MODE_TC_FP16 form); results to host_out, the
 * device error word to *status. No reference counterpart. */
ZLFFT_API int zlfft_selftest_tc_dft16(int device, const float* host_in, float* host_out, int* status);

/* ---------------------------------------------------------------- mixed batches
 * Many transforms of different orders and kinds in one call. No reference
 * counterpart: the reference runs one CFFT<F>/RFFT<F> object per length
 * (src/zldsp_fft_cfft.hpp:19, src/zldsp_fft_rfft.hpp:24), so a host program
 * with transforms of several lengths calls forward()/backward() on several
 * objects one after another; here the whole set is one descriptor list. */

/* One transform of a mixed batch. Buffers are device pointers, AoS layout
 * (interleaved complex; RFFT real sides are plain arrays of F), aligned to
 * 2 * sizeof(F); the real output of forward_sqr_mag to sizeof(F). */
typedef struct zlfft_desc {
    int kind;        /* ZLFFT_C2C or ZLFFT_R2C */
    int precision;   /* ZLFFT_F32 or ZLFFT_F64 */
    int order;       /* log2 of the transform length (RFFT: of the real length) */
    int op;          /* ZLFFT_FORWARD, ZLFFT_BACKWARD, ZLFFT_FORWARD_SQR_MAG (RFFT) */
    const void* in;  /* input of this transform */
    void* out;       /* output of this transform; may equal `in` for C2C */
} zlfft_desc;

typedef struct zlfft_mixed_s* zlfft_mixed;

/* schedules of zlfft_mixed_exec */
#define ZLFFT_SCHED_PER_ORDER 0  /* one batched launch per (kind, order, op) group, in a loop */
#define ZLFFT_SCHED_PERSISTENT 1 /* complex orders <= 11 of every group in one persistent launch */
#define ZLFFT_SCHED_GRAPH 2      /* the persistent schedule recorded once into a CUDA graph, replayed */

/* Prepare a mixed batch of n descriptors on `device` (-1: current): plans per
 * (kind, precision, order), the gathered per-transform pointer arrays, the
 * persistent kernel's work list (tiles sorted longest first) and the
 * multi-pass intermediates, all allocated here, so that zlfft_mixed_exec
 * allocates nothing and may be recorded into a CUDA graph. The descriptors
 * are copied; the buffers they point to are used by every exec. The
 * transforms run concurrently, so an output must not overlap another
 * descriptor's output or input (ZLFFT_ERR_INVALID_ARG); inputs may be shared,
 * and out == in runs a transform in place. */
ZLFFT_API int zlfft_mixed_create(zlfft_mixed* mixed, const zlfft_desc* descs, size_t n, int device);

/* Run every transform of the batch on `stream` (a cudaStream_t; NULL = the
 * legacy default stream), asynchronously, with the given ZLFFT_SCHED_*.
 * Results are identical across schedules. Calls on one mixed object must not
 * overlap on the GPU (they share its work-list counter and intermediates). */
ZLFFT_API int zlfft_mixed_exec(zlfft_mixed mixed, int schedule, void* stream);

/* Number of CUDA kernels the batch's executions have launched since the
 * previous call (a graph replay counts the kernels it contains). */
ZLFFT_API int zlfft_mixed_take_launch_count(zlfft_mixed mixed, size_t* launches);

/* zlfft_plan_device_status over every plan of the batch. */
ZLFFT_API int zlfft_mixed_device_status(zlfft_mixed mixed, int* status);

ZLFFT_API int zlfft_mixed_destroy(zlfft_mixed mixed);

/* One-shot form: create, run with ZLFFT_SCHED_PERSISTENT on `stream`,
 * synchronise the stream, destroy. */
ZLFFT_API int zlfft_exec_mixed_device(const zlfft_desc* descs, size_t n, void* stream);

/* ---------------------------------------------------------------- autotuning
 * No reference counterpart: the reference picks its algorithm from the host
 * CPU's cache sizes (src/common/zldsp_fft_common_system.hpp:132-157); here the
 * plan of each transform size is chosen by measurement on the device.
 *
 * Tuned parameters: for the multi-pass sizes (complex order >= 14) the scratch
 * chunk per pipeline, one or two chunk pipelines, TMA staging or direct loads
 * of the pass inputs, the first pass's output by TMA tensor stores or copied
 * out by the threads, for RFFT forward the split as its own kernel or fused
 * into the last pass, and the computation form (plain, fast-twiddle, and for
 * CFFT<float> the tensor-core split form); for the single-tile sizes, TMA staging or direct
 * loads. None of them changes the arithmetic of a form. Every plan created
 * afterwards on that device and size uses the tuned chunk, pipelines and
 * staging; plans created with ZLFFT_MODE_TUNED also take the tuned form
 * (without a tuning entry they behave as ZLFFT_MODE_PLAIN). Mixed batches
 * create their plans with ZLFFT_MODE_TUNED. If the environment variable
 * ZLFFT_TUNE_FILE names a file written by zlfft_tuning_save, the first plan
 * created on a device loads it. */
typedef struct zlfft_tuning {
    int chunk_mb;       /* scratch per chunk pipeline buffer, MiB (0: single-tile size) */
    int streams;        /* chunk pipelines, 1 or 2 */
    int tma;            /* 1: inputs staged by TMA copies; 0: direct loads */
    int form;           /* ZLFFT_MODE_PLAIN, ZLFFT_MODE_FAST or ZLFFT_MODE_TC_FP16 */
    int split_fused;    /* RFFT forward: 1 = split fused into the last pass, 0 = its own kernel */
    int store_tma;      /* first pass: 1 = output by TMA tensor stores, 0 = copied out, -1 = default */
    double gbs;         /* measured algorithmic GB/s of the chosen plan (forward, AoS) */
    double gbs_default; /* of the default plan (48 MiB, 2 pipelines, TMA, plain) */
} zlfft_tuning;

/* Measure the candidate plans of every order in [order_lo, order_hi] for
 * (kind, precision) on `device` (-1: current), forward AoS -> AoS on about
 * 512 MiB of device buffers allocated for the duration, and record the
 * fastest in the process's tuning table (replacing older entries). Takes
 * about a second per multi-pass order. */
ZLFFT_API int zlfft_autotune(int device, int kind, int precision, size_t order_lo, size_t order_hi);

/* The tuning entry of (device, kind, precision, order); ZLFFT_ERR_UNSUPPORTED
 * if there is none. */
ZLFFT_API int zlfft_tuning_get(int device, int kind, int precision, size_t order, zlfft_tuning* out);

/* Write the device's tuning entries to a text file, headed by the GPU's name
 * and SM count; load such a file into the table (entries written on a GPU of
 * another name or SM count are skipped). *loaded = entries taken. */
ZLFFT_API int zlfft_tuning_save(int device, const char* path);
ZLFFT_API int zlfft_tuning_load(int device, const char* path, size_t* loaded);

/* Forget every tuning entry of every device. */
ZLFFT_API int zlfft_tuning_clear(void);

/* Message of the calling thread's last failure ("" if none). */
ZLFFT_API const char* zlfft_last_error(void);

/* Library version string. */
ZLFFT_API const char* zlfft_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ZLFFT_H_ */
