/* TEST INFRASTRUCTURE ONLY — body of the scalar restatement, instantiated
 * twice by zlfft_oracle.c (float and double). See that file's header.
 *
 * Expects: ZLO_F (scalar type), ZLO_SUF(name) (suffixing macro), ZLO_FMA.
 */

typedef struct {
    ZLO_F r, i;
} ZLO_SUF(cpx);

#define CPX ZLO_SUF(cpx)

/* 1/sqrt(2) as the reference forms it: the double quotient, rounded to F
 * (src/common/zldsp_fft_common_radix.hpp:495). */
static const ZLO_F ZLO_SUF(k_inv_sqrt2) = (ZLO_F)(1.0 / 1.4142135623730951);

/* Twiddle table T[t] = exp(-2*pi*i*t/N), t in [0, 3N/4), each part computed in
 * double as cos(a*pi) / sin(a*pi) with a = -2t/N, then rounded to F.
 * Follows src/common/zldsp_fft_common_init.hpp:138-162 and
 * src/common/zldsp_fft_common_math.hpp:19-24: the reference's per-stage value
 * for (stage width L, multiplier m, index k) is cospi(k * (-2/(4L)) * m); that
 * double equals -2t/N exactly for t = m*k*N/(4L), so one table serves all
 * stages with identical bits. */
void ZLO_SUF(zlo_twiddles)(size_t order, ZLO_F* re, ZLO_F* im) {
    const size_t n = (size_t)1 << order;
    const size_t count = (3 * n) / 4;
    for (size_t t = 0; t < count; ++t) {
        const double a = (double)t * (-2.0 / (double)n);
        re[t] = (ZLO_F)cos(a * M_PI);
        im[t] = (ZLO_F)sin(a * M_PI);
    }
}

/* RFFT split twiddles for k = 1..M/2 (M = N/2 complex points):
 * wc[k] = 0.5*cos(2*pi*k/N), ws[k] = 0.5*sin(2*pi*k/N) + 0.5, in double then
 * rounded (src/common/zldsp_fft_common_init.hpp:374-381). Index 0 unused. */
void ZLO_SUF(zlo_rfft_twiddles)(size_t rfft_order, ZLO_F* wc, ZLO_F* ws) {
    const size_t nr = (size_t)1 << rfft_order;
    const size_t m = nr / 2;
    const double step = 2.0 / (double)nr;
    wc[0] = 0;
    ws[0] = 0;
    for (size_t k = 1; k <= m / 2; ++k) {
        const double a = (double)k * step;
        wc[k] = (ZLO_F)(0.5 * cos(a * M_PI));
        ws[k] = (ZLO_F)(0.5 * sin(a * M_PI) + 0.5);
    }
}

/* x * w with the reference's rounding: re = fma(-xi, wi, xr*wr), im = fma(xi, wr, xr*wi)
 * (src/common/zldsp_fft_common_radix.hpp:114-115). */
static inline CPX ZLO_SUF(cmul)(CPX x, CPX w) {
    CPX t;
    t.r = ZLO_FMA(-x.i, w.i, x.r * w.r);
    t.i = ZLO_FMA(x.i, w.r, x.r * w.i);
    return t;
}

/* First Stockham pass, radix 4, no twiddles: sub-transforms of length 1 -> 4.
 * y[4j+m] = DFT4 over x[j + q*N/4]  (src/common/zldsp_fft_common_radix.hpp:170-239). */
static void ZLO_SUF(pass_first4)(size_t n, const CPX* x, CPX* y) {
    const size_t q = n / 4;
    for (size_t j = 0; j < q; ++j) {
        const CPX a = x[j], b = x[j + q], c = x[j + 2 * q], d = x[j + 3 * q];
        const CPX t0 = {a.r + c.r, a.i + c.i}, t1 = {a.r - c.r, a.i - c.i};
        const CPX t2 = {b.r + d.r, b.i + d.i}, t3 = {b.r - d.r, b.i - d.i};
        y[4 * j + 0] = (CPX){t0.r + t2.r, t0.i + t2.i};
        y[4 * j + 1] = (CPX){t1.r + t3.i, t1.i - t3.r};
        y[4 * j + 2] = (CPX){t0.r - t2.r, t0.i - t2.i};
        y[4 * j + 3] = (CPX){t1.r - t3.i, t1.i + t3.r};
    }
}

/* First Stockham pass, radix 8, no table twiddles (the internal W8 factors use
 * 1/sqrt(2)): sub-transforms of length 1 -> 8. y[8j+p] = DFT8 over x[j + q*N/8]
 * (src/common/zldsp_fft_common_radix.hpp:477-657, kernel.hpp:84-144). */
static void ZLO_SUF(pass_first8)(size_t n, const CPX* x, CPX* y) {
    const size_t e = n / 8;
    const ZLO_F c = ZLO_SUF(k_inv_sqrt2);
    for (size_t j = 0; j < e; ++j) {
        CPX a = x[j], b = x[j + 4 * e];
        const CPX t0 = {a.r + b.r, a.i + b.i}, t1 = {a.r - b.r, a.i - b.i};
        a = x[j + 2 * e];
        b = x[j + 6 * e];
        const CPX t2 = {a.r + b.r, a.i + b.i}, t3 = {a.r - b.r, a.i - b.i};
        const CPX y00 = {t0.r + t2.r, t0.i + t2.i}, y02 = {t0.r - t2.r, t0.i - t2.i};
        const CPX y01 = {t1.r + t3.i, t1.i - t3.r}, y03 = {t1.r - t3.i, t1.i + t3.r};
        a = x[j + e];
        b = x[j + 5 * e];
        const CPX u0 = {a.r + b.r, a.i + b.i}, u1 = {a.r - b.r, a.i - b.i};
        a = x[j + 3 * e];
        b = x[j + 7 * e];
        const CPX u2 = {a.r + b.r, a.i + b.i}, u3 = {a.r - b.r, a.i - b.i};
        const CPX y10 = {u0.r + u2.r, u0.i + u2.i}, y12 = {u0.r - u2.r, u0.i - u2.i};
        const CPX y11 = {u1.r + u3.i, u1.i - u3.r}, y13 = {u1.r - u3.i, u1.i + u3.r};
        const CPX v1 = {(y11.r + y11.i) * c, (y11.i - y11.r) * c};
        const CPX v2 = {y12.i, -y12.r};
        const CPX v3 = {(y13.i - y13.r) * c, (-(y13.r + y13.i)) * c};
        CPX* o = y + 8 * j;
        o[0] = (CPX){y00.r + y10.r, y00.i + y10.i};
        o[1] = (CPX){y01.r + v1.r, y01.i + v1.i};
        o[2] = (CPX){y02.r + v2.r, y02.i + v2.i};
        o[3] = (CPX){y03.r + v3.r, y03.i + v3.i};
        o[4] = (CPX){y00.r - y10.r, y00.i - y10.i};
        o[5] = (CPX){y01.r - v1.r, y01.i - v1.i};
        o[6] = (CPX){y02.r - v2.r, y02.i - v2.i};
        o[7] = (CPX){y03.r - v3.r, y03.i - v3.i};
    }
}

/* Stockham radix-4 DIT pass: sub-transforms of length L -> 4L.
 * Inputs x[i + q*N/4] (i = j*L + k), twiddled by W_{4L}^{q*k} = T[(q*k) << s]
 * with N/(4L) = 1 << s; outputs y[j*4L + k + m*L]
 * (src/common/zldsp_fft_common_radix.hpp:78-158, :391-465). */
static void ZLO_SUF(pass_r4)(size_t n, size_t L, const CPX* x, CPX* y, const CPX* tw, unsigned s) {
    const size_t q = n / 4;
    for (size_t i = 0; i < q; ++i) {
        const size_t k = i % L, j = i / L;
        const CPX t1 = ZLO_SUF(cmul)(x[i + q], tw[(1 * k) << s]);
        const CPX t3 = ZLO_SUF(cmul)(x[i + 3 * q], tw[(3 * k) << s]);
        const CPX s2 = {t1.r + t3.r, t1.i + t3.i}, s3 = {t1.r - t3.r, t1.i - t3.i};
        const CPX t2 = ZLO_SUF(cmul)(x[i + 2 * q], tw[(2 * k) << s]);
        const CPX x0 = x[i];
        const CPX s0 = {x0.r + t2.r, x0.i + t2.i}, s1 = {x0.r - t2.r, x0.i - t2.i};
        CPX* o = y + j * 4 * L + k;
        o[0] = (CPX){s0.r + s2.r, s0.i + s2.i};
        o[L] = (CPX){s1.r + s3.i, s1.i - s3.r};
        o[2 * L] = (CPX){s0.r - s2.r, s0.i - s2.i};
        o[3 * L] = (CPX){s1.r - s3.i, s1.i + s3.r};
    }
}

/* Forward DFT of x (length 1<<order) into y, in the reference's stage order:
 * radix-8 first pass for odd orders >= 3, radix-4 first pass for even orders
 * >= 2, then radix-4 passes L = 4 or 8, x4 each, up to N
 * (src/common/zldsp_fft_common_init.hpp:193-206, execute.hpp:26-144,
 * kernel.hpp:19-144). x is clobbered. tw is the unified table of a length
 * 2^tshift times N; entry t << tshift of it equals entry t of this order's own
 * table bit for bit (the same double argument a = -2t/N, the exact power-of-two
 * scaling cancels). */
static void ZLO_SUF(dft_forward_t)(size_t order, CPX* x, CPX* y, const CPX* tw, unsigned tshift);
static void ZLO_SUF(dft_forward)(size_t order, CPX* x, CPX* y, const CPX* tw) {
    ZLO_SUF(dft_forward_t)(order, x, y, tw, 0);
}
static void ZLO_SUF(dft_forward_t)(size_t order, CPX* x, CPX* y, const CPX* tw, unsigned tshift) {
    const size_t n = (size_t)1 << order;
    if (order == 0) {
        y[0] = x[0];
        return;
    }
    if (order == 1) {
        y[0] = (CPX){x[0].r + x[1].r, x[0].i + x[1].i};
        y[1] = (CPX){x[0].r - x[1].r, x[0].i - x[1].i};
        return;
    }
    size_t L;
    if (order % 2) {
        ZLO_SUF(pass_first8)(n, x, y);
        L = 8;
    } else {
        ZLO_SUF(pass_first4)(n, x, y);
        L = 4;
    }
    CPX* cur = y;
    CPX* nxt = x;
    unsigned s = 0;
    while ((n >> s) > 4 * L) ++s; /* n / (4L) = 1 << s */
    while (L < n) {
        ZLO_SUF(pass_r4)(n, L, cur, nxt, tw, s + tshift);
        CPX* t = cur;
        cur = nxt;
        nxt = t;
        L *= 4;
        s = s >= 2 ? s - 2 : 0;
    }
    if (cur != y) memcpy(y, cur, n * sizeof(CPX));
}

/* ---------------------------------------------------------------- macro path
 * The reference's algorithm switch (src/common/zldsp_fft_common_init.hpp:305-339):
 * a CFFT of order >= switch_order runs as Cooley-Tukey DIF macro stages, then
 * a micro Stockham FFT per segment, then a digit-reversed transposed store.
 * The micro order is max_l1_order, or max_l1_order - 1 when order - max_l1_order
 * is odd, so the macro stages are radix-4. The values come from the host's
 * cache sizes in the reference (src/common/zldsp_fft_common_system.hpp:132-157);
 * here the caller sets them. Default: never (micro-only), the reference's
 * choice on a host whose caches put switch_order above every order used. */
static int ZLO_SUF(g_max_l1) = 0;
static int ZLO_SUF(g_switch) = 1 << 30;

void ZLO_SUF(zlo_set_hybrid)(int max_l1_order, int switch_order) {
    ZLO_SUF(g_max_l1) = max_l1_order;
    ZLO_SUF(g_switch) = switch_order;
}

/* Micro order of the macro path for `order`, or -1 for the micro-only path. */
int ZLO_SUF(zlo_micro_order)(size_t order) {
    if ((long)order < (long)ZLO_SUF(g_switch)) return -1;
    const int l1 = ZLO_SUF(g_max_l1);
    return ((long)order - l1) % 2 != 0 ? l1 - 1 : l1;
}

/* One radix-4 DIF stage in place, butterfly stride w: for each block of 4w
 * points and j < w, x[j + q*w] (q = 0..3) -> DFT4 with the twiddle W_{4w}^{m j}
 * applied to output m AFTER the butterfly; outputs stay at their positions
 * (src/common/zldsp_fft_common_radix.hpp:670-751 first stage with the loads,
 * :762-843 the in-place stages). The twiddle of the reference's stage table
 * (init.hpp:227-274: cospi(m * j * (-2/(4w)))) is entry (m*j) << s of the
 * unified table, n/(4w) = 1 << s. */
static void ZLO_SUF(dif_stage)(size_t n, size_t w, CPX* x, const CPX* tw, unsigned s) {
    for (size_t blk = 0; blk < n; blk += 4 * w) {
        CPX* p = x + blk;
        for (size_t j = 0; j < w; ++j) {
            const CPX a = p[j], b = p[j + w], c = p[j + 2 * w], d = p[j + 3 * w];
            const CPX t0 = {a.r + c.r, a.i + c.i}, t1 = {a.r - c.r, a.i - c.i};
            const CPX t2 = {b.r + d.r, b.i + d.i}, t3 = {b.r - d.r, b.i - d.i};
            const CPX y0 = {t0.r + t2.r, t0.i + t2.i};
            const CPX y2 = {t0.r - t2.r, t0.i - t2.i};
            const CPX y1 = {t1.r + t3.i, t1.i - t3.r};
            const CPX y3 = {t1.r - t3.i, t1.i + t3.r};
            p[j] = y0;
            p[j + w] = ZLO_SUF(cmul)(y1, tw[(1 * j) << s]);
            p[j + 2 * w] = ZLO_SUF(cmul)(y2, tw[(2 * j) << s]);
            p[j + 3 * w] = ZLO_SUF(cmul)(y3, tw[(3 * j) << s]);
        }
    }
}

/* Base-4 digit reversal of c over nd digits (init.hpp:282-296). */
static size_t ZLO_SUF(digit_rev4)(size_t c, size_t nd) {
    size_t r = 0;
    for (size_t d = 0; d < nd; ++d) {
        r = (r << 2) | (c & 3);
        c >>= 2;
    }
    return r;
}

/* Forward macro-path DFT of a (length 1<<order, already direction-swapped),
 * clobbering a; output element k*S + c (S = segments) goes to (re, im, step)
 * through the store swap (src/common/zldsp_fft_common_execute.hpp:174-272):
 * column c is the micro FFT of the segment at digit_rev4(c). b is scratch of
 * at least 2 * 2^micro points. */
static void ZLO_SUF(macro_forward)(size_t order, int micro, int forward, const CPX* tw, CPX* a, CPX* b,
                                   ZLO_F* out_re, ZLO_F* out_im, size_t out_step) {
    const size_t n = (size_t)1 << order;
    const size_t nm = (order - (size_t)micro) / 2;
    for (size_t i = 0; i < nm; ++i) ZLO_SUF(dif_stage)(n, n >> (2 * i + 2), a, tw, (unsigned)(2 * i));
    const size_t m = (size_t)1 << micro, segs = n >> micro;
    for (size_t c = 0; c < segs; ++c) {
        memcpy(b, a + ZLO_SUF(digit_rev4)(c, nm) * m, m * sizeof(CPX));
        ZLO_SUF(dft_forward_t)((size_t)micro, b, b + m, tw, (unsigned)(order - (size_t)micro));
        const CPX* y = b + m;
        for (size_t k = 0; k < m; ++k) {
            const size_t o = (k * segs + c) * out_step;
            out_re[o] = forward ? y[k].r : y[k].i;
            out_im[o] = forward ? y[k].i : y[k].r;
        }
    }
}

/* Complex FFT of one transform with the reference's conventions:
 * forward = DFT with exp(-i...), backward = swap(DFT(swap(x))) = unnormalised
 * inverse (src/common/zldsp_fft_common_structure.hpp:47-135).
 * Layout is given by (re, im, step): AoS is (p, p+1, 2), SoA is (r, i, 1).
 * tw is the table of zlo_twiddles(order); a and b are scratch of N points.
 * Orders at or above the switch take the macro path (zlo_set_hybrid). */
static void ZLO_SUF(cfft_core)(size_t order, int forward, const CPX* tw, const ZLO_F* in_re, const ZLO_F* in_im,
                               size_t in_step, ZLO_F* out_re, ZLO_F* out_im, size_t out_step, CPX* a, CPX* b) {
    const size_t n = (size_t)1 << order;
    for (size_t k = 0; k < n; ++k) {
        const ZLO_F r = in_re[k * in_step], i = in_im[k * in_step];
        a[k] = forward ? (CPX){r, i} : (CPX){i, r};
    }
    const int micro = ZLO_SUF(zlo_micro_order)(order);
    if (micro >= 0 && (size_t)micro + 2 <= order) {
        ZLO_SUF(macro_forward)(order, micro, forward, tw, a, b, out_re, out_im, out_step);
        return;
    }
    ZLO_SUF(dft_forward)(order, a, b, tw);
    for (size_t k = 0; k < n; ++k) {
        out_re[k * out_step] = forward ? b[k].r : b[k].i;
        out_im[k * out_step] = forward ? b[k].i : b[k].r;
    }
}

static CPX* ZLO_SUF(make_table)(size_t order) {
    const size_t n = (size_t)1 << order;
    const size_t nt = (3 * n) / 4 + 1;
    ZLO_F* twr = (ZLO_F*)malloc(nt * sizeof(ZLO_F));
    ZLO_F* twi = (ZLO_F*)malloc(nt * sizeof(ZLO_F));
    CPX* tw = (CPX*)malloc(nt * sizeof(CPX));
    ZLO_SUF(zlo_twiddles)(order, twr, twi);
    for (size_t t = 0; t < (3 * n) / 4; ++t) tw[t] = (CPX){twr[t], twi[t]};
    free(twr);
    free(twi);
    return tw;
}

void ZLO_SUF(zlo_cfft)(size_t order, int forward, const ZLO_F* in_re, const ZLO_F* in_im, size_t in_step,
                       ZLO_F* out_re, ZLO_F* out_im, size_t out_step) {
    const size_t n = (size_t)1 << order;
    CPX* a = (CPX*)malloc(n * sizeof(CPX));
    CPX* b = (CPX*)malloc(n * sizeof(CPX));
    CPX* tw = ZLO_SUF(make_table)(order);
    ZLO_SUF(cfft_core)(order, forward, tw, in_re, in_im, in_step, out_re, out_im, out_step, a, b);
    free(a);
    free(b);
    free(tw);
}

/* A batch of complex transforms (layout codes: 0 AoS, 1 SoA; transform b at
 * offset b*N complex values), split over nthreads POSIX threads. */
typedef struct {
    size_t order, b0, b1;
    int forward, in_layout, out_layout;
    const ZLO_F *in_re, *in_im;
    ZLO_F *out_re, *out_im;
    const CPX* tw;
} ZLO_SUF(cfft_job);

static void* ZLO_SUF(cfft_worker)(void* arg) {
    const ZLO_SUF(cfft_job)* jb = (const ZLO_SUF(cfft_job)*)arg;
    const size_t n = (size_t)1 << jb->order;
    CPX* a = (CPX*)malloc(n * sizeof(CPX));
    CPX* b = (CPX*)malloc(n * sizeof(CPX));
    for (size_t t = jb->b0; t < jb->b1; ++t) {
        const ZLO_F *ir, *ii;
        ZLO_F *orr, *oi;
        size_t is, os;
        if (jb->in_layout == 0) {
            ir = jb->in_re + 2 * n * t;
            ii = ir + 1;
            is = 2;
        } else {
            ir = jb->in_re + n * t;
            ii = jb->in_im + n * t;
            is = 1;
        }
        if (jb->out_layout == 0) {
            orr = jb->out_re + 2 * n * t;
            oi = orr + 1;
            os = 2;
        } else {
            orr = jb->out_re + n * t;
            oi = jb->out_im + n * t;
            os = 1;
        }
        ZLO_SUF(cfft_core)(jb->order, jb->forward, jb->tw, ir, ii, is, orr, oi, os, a, b);
    }
    free(a);
    free(b);
    return NULL;
}

void ZLO_SUF(zlo_cfft_batch)(size_t order, int forward, int in_layout, const ZLO_F* in_re, const ZLO_F* in_im,
                             int out_layout, ZLO_F* out_re, ZLO_F* out_im, size_t batch, int nthreads) {
    CPX* tw = ZLO_SUF(make_table)(order);
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > batch) nthreads = batch ? (int)batch : 1;
    pthread_t th[256];
    ZLO_SUF(cfft_job) jobs[256];
    if (nthreads > 256) nthreads = 256;
    size_t start = 0;
    for (int t = 0; t < nthreads; ++t) {
        const size_t cnt = batch / nthreads + ((size_t)t < batch % nthreads ? 1 : 0);
        jobs[t] = (ZLO_SUF(cfft_job)){order, start, start + cnt, forward, in_layout, out_layout,
                                      in_re, in_im, out_re, out_im, tw};
        start += cnt;
        pthread_create(&th[t], NULL, ZLO_SUF(cfft_worker), &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(tw);
}

/* RFFT forward post-processing from the N/2-point spectrum z of the real
 * input viewed as complex pairs (src/common/zldsp_fft_common_execute.hpp:318-368).
 * mode 0: complex bins to (re, im, step); mode 1: squared magnitudes to out_re
 * (execute.hpp:481-536). Bins k and M-k come from one pair; at k = M/2 the
 * reference's second store (the M-k formula) is the one that remains. */
static void ZLO_SUF(rfft_post)(size_t m, const CPX* z, const ZLO_F* wc, const ZLO_F* ws, int mode,
                               ZLO_F* out_re, ZLO_F* out_im, size_t step) {
    const ZLO_F r0 = z[0].r, i0 = z[0].i;
    const ZLO_F dc = r0 + i0, ny = r0 - i0;
    if (mode == 0) {
        out_re[0] = dc;
        out_im[0] = 0;
        out_re[m * step] = ny;
        out_im[m * step] = 0;
    } else {
        out_re[0] = dc * dc;
        out_re[m] = ny * ny;
    }
    for (size_t k = 1; k <= m / 2; ++k) {
        const ZLO_F r1 = z[k].r, i1 = z[k].i, r2 = z[m - k].r, i2 = z[m - k].i;
        const ZLO_F c = wc[k], s = ws[k];
        const ZLO_F si = i1 + i2, dr = r1 - r2;
        const ZLO_F xr_k = ZLO_FMA(-dr, s, ZLO_FMA(si, c, r1));
        const ZLO_F xi_k = ZLO_FMA(-dr, c, ZLO_FMA(-si, s, i1));
        const ZLO_F xr_mk = ZLO_FMA(dr, s, ZLO_FMA(-si, c, r2));
        const ZLO_F xi_mk = ZLO_FMA(-dr, c, ZLO_FMA(-si, s, i2));
        if (mode == 0) {
            out_re[k * step] = xr_k;
            out_im[k * step] = xi_k;
            out_re[(m - k) * step] = xr_mk;
            out_im[(m - k) * step] = xi_mk;
        } else {
            out_re[k] = ZLO_FMA(xr_k, xr_k, xi_k * xi_k);
            out_re[m - k] = ZLO_FMA(xr_mk, xr_mk, xi_mk * xi_mk);
        }
    }
}

/* RFFT forward of one real frame of N = 1<<rfft_order samples (rfft_order >= 1).
 * mode 0: N/2+1 complex bins to (out_re, out_im, out_step); mode 1: N/2+1
 * squared magnitudes to out_re (src/zldsp_fft_rfft.hpp:68-109). */
void ZLO_SUF(zlo_rfft_forward)(size_t rfft_order, const ZLO_F* in, int mode, ZLO_F* out_re, ZLO_F* out_im,
                               size_t out_step) {
    const size_t m = (size_t)1 << (rfft_order - 1);
    ZLO_F* z = (ZLO_F*)malloc(2 * m * sizeof(ZLO_F));
    ZLO_F* wc = (ZLO_F*)malloc((m / 2 + 1) * sizeof(ZLO_F));
    ZLO_F* ws = (ZLO_F*)malloc((m / 2 + 1) * sizeof(ZLO_F));
    ZLO_SUF(zlo_rfft_twiddles)(rfft_order, wc, ws);
    ZLO_SUF(zlo_cfft)(rfft_order - 1, 1, in, in + 1, 2, z, z + 1, 2);
    ZLO_SUF(rfft_post)(m, (const CPX*)z, wc, ws, mode, out_re, out_im, out_step);
    free(z);
    free(wc);
    free(ws);
}

/* RFFT backward of N/2+1 bins (layout (in_re, in_im, in_step)) to N reals,
 * unnormalised: forward then backward returns (N/2)*x. Pre-processing follows
 * src/common/zldsp_fft_common_execute.hpp:399-451 (with its 0.5 factors), then
 * an N/2-point backward CFFT (src/zldsp_fft_rfft.hpp:133-137). */
void ZLO_SUF(zlo_rfft_backward)(size_t rfft_order, const ZLO_F* in_re, const ZLO_F* in_im, size_t in_step,
                                ZLO_F* out) {
    const size_t m = (size_t)1 << (rfft_order - 1);
    CPX* z = (CPX*)malloc(m * sizeof(CPX));
    ZLO_F* wc = (ZLO_F*)malloc((m / 2 + 1) * sizeof(ZLO_F));
    ZLO_F* ws = (ZLO_F*)malloc((m / 2 + 1) * sizeof(ZLO_F));
    ZLO_SUF(zlo_rfft_twiddles)(rfft_order, wc, ws);
    const ZLO_F r0 = in_re[0], rm = in_re[m * in_step];
    z[0].r = (r0 + rm) * (ZLO_F)0.5;
    z[0].i = (r0 - rm) * (ZLO_F)0.5;
    for (size_t k = 1; k <= m / 2; ++k) {
        const ZLO_F r1 = in_re[k * in_step], i1 = in_im[k * in_step];
        const ZLO_F r2 = in_re[(m - k) * in_step], i2 = in_im[(m - k) * in_step];
        const ZLO_F c = wc[k], s = ws[k];
        const ZLO_F si = i1 + i2, dr = r1 - r2;
        z[k].r = ZLO_FMA(-dr, s, ZLO_FMA(-si, c, r1));
        z[k].i = ZLO_FMA(dr, c, ZLO_FMA(-si, s, i1));
        z[m - k].r = ZLO_FMA(dr, s, ZLO_FMA(si, c, r2));
        z[m - k].i = ZLO_FMA(dr, c, ZLO_FMA(-si, s, i2));
    }
    ZLO_F* zf = (ZLO_F*)z;
    ZLO_SUF(zlo_cfft)(rfft_order - 1, 0, zf, zf + 1, 2, out, out + 1, 2);
    free(z);
    free(wc);
    free(ws);
}

#undef CPX
