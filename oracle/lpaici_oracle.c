/*
 * lpaici_oracle.c -- CPU restatement of the reference LPA-ICI path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the oracle.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * may load it, and only as the checker; the product library never links or calls it.
 *
 * What it restates (titocapovilla/lpa-ici-cuda, paths relative to that project):
 *   oracle_load_kernels   <- load_LPA_kernels_standardized   src/v1_0_lpa_ici_2D_fused.cpp:466-551
 *   oracle_variances      <- compute_kernel_variances        src/v1_0_lpa_ici_2D_fused.cpp:691-717
 *   oracle_pack_runs      <- build_sparse_kernels            src/v4_1_lpa_ici_2D_sparse_shared.cu:826-877
 *   oracle_forward_f32    <- anisotropic_lpa_ici_cpu_fused   src/v1_0_lpa_ici_2D_fused.cpp:851-930
 *                            + process_scale_fused           src/v1_0_lpa_ici_2D_fused.cpp:803-849
 *   oracle_psnr           <- calculate_PSNR                  src/v1_0_lpa_ici_2D_fused.cpp:778-799
 * and, with no counterpart in the reference, FP64 restatements used to state errors and to check
 * the adjoint: oracle_forward_f64, oracle_adjoint_f64 (selection frozen) and
 * oracle_fd_grad_f64 (central finite differences of the frozen-selection map).
 *
 * Arithmetic.  The reference's CPU build (g++ -O3, x86-64 without -march) rounds every multiply
 * and every add separately and sums the taps of a kernel in row-major order.  This file is built
 * with -ffp-contract=off and keeps that order.  It visits only the nonzero taps: starting from
 * +0.0f, a running sum can never become -0.0f, and adding +-0.0f to any other value returns it
 * unchanged, so skipping the zero taps leaves every bit of a finite result unchanged while doing
 * 5 % of the dense work.  (For non-finite inputs the dense reference turns 0*inf into NaN; that
 * case is outside the oracle.)
 *
 * Pinning: tests/test_oracle_pin.py checks every function here bit-for-bit against the reference's
 * own functions compiled in-process from its sources (oracle/Makefile -> oracle/_ref/), and against
 * the fixtures in tests/golden/ that those functions produced (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------------------------ */
/* Kernel file loader (load_LPA_kernels_standardized, v1_0_lpa_ici_2D_fused.cpp:466-551).       */
/* ------------------------------------------------------------------------------------------ */

/* A character stream over the whole file, read the way std::istream's operator>> reads numbers in
 * the "C" locale: skip whitespace, take the longest numeric prefix, leave the rest for the next read.
 * Integers [+-]?[0-9]+; floats [+-]?[0-9]*(.[0-9]*)?([eE][+-]?[0-9]+)? with a mantissa digit, converted
 * by strtof (correctly rounded, as libstdc++ converts); overflow and a digitless exponent fail. */
typedef struct {
    const char *p, *end;
} stream_t;

static int is_space(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }
static int is_digit(char c) { return c >= '0' && c <= '9'; }

static int next_int(stream_t *s, int *v) {
    while (s->p < s->end && is_space(*s->p)) s->p++;
    const char *b = s->p;
    if (s->p < s->end && (*s->p == '+' || *s->p == '-')) s->p++;
    const char *d = s->p;
    while (s->p < s->end && is_digit(*s->p)) s->p++;
    if (s->p == d || s->p - b > 15) return 0;
    char buf[32];
    memcpy(buf, b, (size_t)(s->p - b));
    buf[s->p - b] = '\0';
    long x = strtol(buf, NULL, 10);
    if (x > 2147483647L || x < -2147483648L) return 0;
    *v = (int)x;
    return 1;
}

static int next_float(stream_t *s, float *v) {
    while (s->p < s->end && is_space(*s->p)) s->p++;
    const char *b = s->p;
    int mant = 0;
    if (s->p < s->end && (*s->p == '+' || *s->p == '-')) s->p++;
    while (s->p < s->end && is_digit(*s->p)) s->p++, mant++;
    if (s->p < s->end && *s->p == '.') {
        s->p++;
        while (s->p < s->end && is_digit(*s->p)) s->p++, mant++;
    }
    if (!mant) return 0;
    if (s->p < s->end && (*s->p == 'e' || *s->p == 'E')) {
        int ed = 0;
        s->p++;
        if (s->p < s->end && (*s->p == '+' || *s->p == '-')) s->p++;
        while (s->p < s->end && is_digit(*s->p)) s->p++, ed++;
        if (!ed) return 0;
    }
    size_t n = (size_t)(s->p - b);
    char *buf = (char *)malloc(n + 1);
    memcpy(buf, b, n);
    buf[n] = '\0';
    char *e;
    *v = strtof(buf, &e);
    int ok = *e == '\0' && !isinf(*v);
    free(buf);
    return ok;
}

/* Returns 0 on success, 1 when the file cannot be opened, 2 on malformed content.
 * On success *w (size sum rows*cols), *off, *rows, *cols (size D*S) are malloc'd; free with
 * oracle_free.  Every direction is centre-cropped to direction 0's size at the same scale,
 * the crop offset being (file - target) / 2 (v1_0_lpa_ici_2D_fused.cpp:511-543).  A kernel
 * smaller than the target is rejected here; the reference only rejects a negative offset and
 * would read outside its buffer for an odd size difference. */
ORACLE_API int oracle_load_kernels(const char *path, int *D_out, int *S_out, float **w_out, int **off_out,
                                   int **rows_out, int **cols_out) {
    FILE *f = fopen(path, "rb");
    if (!f) return 1;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *text = (char *)malloc((size_t)n + 1);
    size_t len = fread(text, 1, (size_t)n, f);
    text[len] = '\0';
    fclose(f);
    stream_t st = {text, text + len}, *t = &st;

    int D, S, rc = 2;
    float *w = NULL, *tmp = NULL;
    int *off = NULL, *rows = NULL, *cols = NULL, *trow = NULL, *tcol = NULL;
    size_t wcap = 0, wlen = 0;
    if (!next_int(t, &D) || !next_int(t, &S) || D <= 0 || S <= 0) goto done;
    off = (int *)malloc(sizeof(int) * D * S);
    rows = (int *)malloc(sizeof(int) * D * S);
    cols = (int *)malloc(sizeof(int) * D * S);
    trow = (int *)malloc(sizeof(int) * S);
    tcol = (int *)malloc(sizeof(int) * S);
    for (int d = 0; d < D; d++) {
        for (int s = 0; s < S; s++) {
            int fr, fc;
            if (!next_int(t, &fr) || !next_int(t, &fc) || fr <= 0 || fc <= 0) goto done;
            size_t ne = (size_t)fr * fc;
            tmp = (float *)realloc(tmp, sizeof(float) * ne);
            for (size_t i = 0; i < ne; i++)
                if (!next_float(t, &tmp[i])) goto done;
            if (d == 0) {
                trow[s] = fr;
                tcol[s] = fc;
            }
            int tr = trow[s], tc = tcol[s];
            if (fr < tr || fc < tc) goto done;
            int ro = (fr - tr) / 2, co = (fc - tc) / 2;
            int k = d * S + s;
            off[k] = (int)wlen;
            rows[k] = tr;
            cols[k] = tc;
            if (wlen + (size_t)tr * tc > wcap) {
                wcap = (wlen + (size_t)tr * tc) * 2;
                w = (float *)realloc(w, sizeof(float) * wcap);
            }
            for (int r = 0; r < tr; r++)
                for (int c = 0; c < tc; c++) w[wlen++] = tmp[(size_t)(r + ro) * fc + (c + co)];
        }
    }
    rc = 0;
done:
    free(text);
    free(tmp);
    free(trow);
    free(tcol);
    if (rc != 0) {
        free(w);
        free(off);
        free(rows);
        free(cols);
        return rc;
    }
    *D_out = D;
    *S_out = S;
    *w_out = w;
    *off_out = off;
    *rows_out = rows;
    *cols_out = cols;
    return 0;
}

ORACLE_API void oracle_free(void *p) { free(p); }

/* var[k] = (sigma*sigma) * sum_i w_i*w_i, in float, dense row-major (v1_0...cpp:700-715). */
ORACLE_API void oracle_variances(const float *w, const int *off, const int *rows, const int *cols, int nk,
                                 float sigma, float *var) {
    float s2 = sigma * sigma;
    for (int k = 0; k < nk; k++) {
        float nsq = 0.0f;
        int ne = rows[k] * cols[k];
        for (int i = 0; i < ne; i++) {
            float v = w[off[k] + i];
            nsq += v * v;
        }
        var[k] = s2 * nsq;
    }
}

/* Row runs from the first to the last nonzero of every kernel row, centre-relative, plus the
 * packed weights (build_sparse_kernels, v4_1_lpa_ici_2D_sparse_shared.cu:826-877).  Output arrays
 * must hold at least sum(rows) runs and sum(rows*cols) weights; returns the number of runs and
 * writes the number of weights to *n_weights. */
ORACLE_API int oracle_pack_runs(const float *w, const int *off, const int *rows, const int *cols, int nk,
                                float *weights, int *run_row, int *run_col, int *run_len, int *k_first_run,
                                int *k_num_runs, int *k_first_weight, int *n_weights) {
    int nr = 0, nw = 0;
    for (int k = 0; k < nk; k++) {
        const float *h = w + off[k];
        k_first_run[k] = nr;
        k_first_weight[k] = nw;
        for (int r = 0; r < rows[k]; r++) {
            int first = -1, last = -1;
            for (int c = 0; c < cols[k]; c++)
                if (h[r * cols[k] + c] != 0.0f) {
                    if (first < 0) first = c;
                    last = c;
                }
            if (first < 0) continue;
            run_row[nr] = r - rows[k] / 2;
            run_col[nr] = first - cols[k] / 2;
            run_len[nr] = last - first + 1;
            nr++;
            for (int c = first; c <= last; c++) weights[nw++] = h[r * cols[k] + c];
        }
        k_num_runs[k] = nr - k_first_run[k];
    }
    *n_weights = nw;
    return nr;
}

/* ------------------------------------------------------------------------------------------ */
/* Forward LPA-ICI, FP32, bit-faithful to anisotropic_lpa_ici_cpu_fused.                        */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int dy, dx; /* offset of the tap from the output pixel: (k_row - rows/2, k_col - cols/2) */
    float w;
} tap_t;

/* Nonzero taps of every kernel, row-major, and the per-kernel ranges. */
static tap_t *build_taps(const float *w, const int *off, const int *rows, const int *cols, int nk, int *begin) {
    int total = 0;
    for (int k = 0; k < nk; k++)
        for (int i = 0; i < rows[k] * cols[k]; i++) total += w[off[k] + i] != 0.0f;
    tap_t *taps = (tap_t *)malloc(sizeof(tap_t) * (total > 0 ? total : 1));
    int n = 0;
    for (int k = 0; k < nk; k++) {
        begin[k] = n;
        for (int r = 0; r < rows[k]; r++)
            for (int c = 0; c < cols[k]; c++) {
                float v = w[off[k] + r * cols[k] + c];
                if (v != 0.0f) {
                    taps[n].dy = r - rows[k] / 2;
                    taps[n].dx = c - cols[k] / 2;
                    taps[n].w = v;
                    n++;
                }
            }
    }
    begin[nk] = n;
    return taps;
}

/* out[H*W]            denoised image
 * scale_map[D*H*W]    optional (NULL): index of the last accepted scale per direction and pixel
 * taps_out            optional (NULL): number of nonzero taps the reference's fused loop convolves
 *                     (every scale up to and including the first rejected one, or all S). */
ORACLE_API void oracle_forward_f32(const float *x, int W, int H, int D, int S, const float *w, const int *off,
                                   const int *rows, const int *cols, const float *var, float gamma, float *out,
                                   uint8_t *scale_map, double *taps_out) {
    int nk = D * S;
    int *begin = (int *)malloc(sizeof(int) * (nk + 1));
    tap_t *taps = build_taps(w, off, rows, cols, nk, begin);
    float *thr = (float *)malloc(sizeof(float) * nk);
    for (int k = 0; k < nk; k++) thr[k] = gamma * sqrtf(var[k]); /* v1_0...cpp:905 */
    double ntaps = 0.0;
    size_t npx = (size_t)W * H;
    float *num = (float *)calloc(npx, sizeof(float));
    float *den = (float *)calloc(npx, sizeof(float));
    for (int d = 0; d < D; d++) {
        for (int py = 0; py < H; py++) {
            for (int px = 0; px < W; px++) {
                float lo = -INFINITY, hi = INFINITY, best = 0.0f, bvar = 0.0f;
                int sstar = 0;
                for (int s = 0; s < S; s++) {
                    int k = d * S + s;
                    float conv = 0.0f;
                    for (int t = begin[k]; t < begin[k + 1]; t++) {
                        int iy = py + taps[t].dy, ix = px + taps[t].dx;
                        if (iy >= 0 && iy < H && ix >= 0 && ix < W) conv += taps[t].w * x[(size_t)iy * W + ix];
                    }
                    ntaps += begin[k + 1] - begin[k];
                    float lb = conv - thr[k];
                    float ub = conv + thr[k];
                    lo = lo < lb ? lb : lo; /* std::max(lo, lb) */
                    hi = ub < hi ? ub : hi; /* std::min(hi, ub) */
                    if (hi >= lo) {
                        best = conv;
                        bvar = var[k];
                        sstar = s;
                    } else {
                        break; /* the interval stays empty: v1_0...cpp:815 skips the pixel from now on */
                    }
                }
                size_t p = (size_t)py * W + px;
                num[p] += best * (1.0f / bvar);
                den[p] += 1.0f / bvar;
                if (scale_map) scale_map[(size_t)d * npx + p] = (uint8_t)sstar;
            }
        }
    }
    for (size_t p = 0; p < npx; p++) out[p] = num[p] / den[p];
    if (taps_out) *taps_out = ntaps;
    free(num);
    free(den);
    free(thr);
    free(taps);
    free(begin);
}

/* PSNR in double of a float difference squared in float (v1_0...cpp:778-799). */
ORACLE_API double oracle_psnr(const float *a, const float *b, long n) {
    double sum = 0.0;
    for (long i = 0; i < n; i++) {
        float diff = a[i] - b[i];
        float sq = diff * diff;
        sum += (double)sq;
    }
    double mse = sum / (double)n;
    return 10.0 * log10(1.0f / mse);
}

/* Algorithmic tap count from a scale map: for every (direction, pixel) the taps of scales
 * 0..min(s*+1, S-1), i.e. the scales the fused reference convolves. */
ORACLE_API double oracle_count_taps(const uint8_t *scale_map, long npx, int D, int S, const int *nnz) {
    double total = 0.0;
    for (int d = 0; d < D; d++) {
        double prefix[257];
        prefix[0] = 0.0;
        for (int s = 0; s < S; s++) prefix[s + 1] = prefix[s] + nnz[d * S + s];
        const uint8_t *m = scale_map + (size_t)d * npx;
        for (long p = 0; p < npx; p++) {
            int stop = m[p] + 1 < S ? m[p] + 1 : S - 1;
            total += prefix[stop + 1];
        }
    }
    return total;
}

/* ------------------------------------------------------------------------------------------ */
/* FP64 restatements (no reference counterpart): error statements and the adjoint check.        */
/* ------------------------------------------------------------------------------------------ */

/* The same algorithm in double: variances sigma^2 * sum w^2 and thresholds gamma * sqrt(var)
 * in double from the float weights; ICI decisions in double. */
ORACLE_API void oracle_forward_f64(const float *x, int W, int H, int D, int S, const float *w, const int *off,
                                   const int *rows, const int *cols, double sigma, double gamma, double *out,
                                   uint8_t *scale_map) {
    int nk = D * S;
    int *begin = (int *)malloc(sizeof(int) * (nk + 1));
    tap_t *taps = build_taps(w, off, rows, cols, nk, begin);
    double *var = (double *)malloc(sizeof(double) * nk), *thr = (double *)malloc(sizeof(double) * nk);
    for (int k = 0; k < nk; k++) {
        double nsq = 0.0;
        for (int i = 0; i < rows[k] * cols[k]; i++) nsq += (double)w[off[k] + i] * (double)w[off[k] + i];
        var[k] = sigma * sigma * nsq;
        thr[k] = gamma * sqrt(var[k]);
    }
    size_t npx = (size_t)W * H;
    double *num = (double *)calloc(npx, sizeof(double)), *den = (double *)calloc(npx, sizeof(double));
    for (int d = 0; d < D; d++)
        for (int py = 0; py < H; py++)
            for (int px = 0; px < W; px++) {
                double lo = -INFINITY, hi = INFINITY, best = 0.0, bvar = 0.0;
                int sstar = 0;
                for (int s = 0; s < S; s++) {
                    int k = d * S + s;
                    double conv = 0.0;
                    for (int t = begin[k]; t < begin[k + 1]; t++) {
                        int iy = py + taps[t].dy, ix = px + taps[t].dx;
                        if (iy >= 0 && iy < H && ix >= 0 && ix < W) conv += (double)taps[t].w * x[(size_t)iy * W + ix];
                    }
                    lo = fmax(lo, conv - thr[k]);
                    hi = fmin(hi, conv + thr[k]);
                    if (hi >= lo) {
                        best = conv;
                        bvar = var[k];
                        sstar = s;
                    } else
                        break;
                }
                size_t p = (size_t)py * W + px;
                num[p] += best / bvar;
                den[p] += 1.0 / bvar;
                if (scale_map) scale_map[(size_t)d * npx + p] = (uint8_t)sstar;
            }
    for (size_t p = 0; p < npx; p++) out[p] = num[p] / den[p];
    free(num);
    free(den);
    free(var);
    free(thr);
    free(taps);
    free(begin);
}

/* Aggregation weights alpha_d(p) = (1/v_d(p)) / sum_d' (1/v_d'(p)) of a frozen selection, in
 * double, with v_d(p) = var[d, s*(d,p)] (var given in float, as the forward uses it). */
static void frozen_alpha(const uint8_t *smap, size_t npx, int D, int S, const float *var, size_t p, double *alpha) {
    double den = 0.0;
    for (int d = 0; d < D; d++) {
        alpha[d] = 1.0 / (double)var[d * S + smap[(size_t)d * npx + p]];
        den += alpha[d];
    }
    for (int d = 0; d < D; d++) alpha[d] /= den;
}

/* Adjoint of the frozen-selection map x -> out, in double:
 *   grad[q] = sum_d sum_p g[p] * alpha_d(p) * h_{d,s*(d,p)}(q - p + c)      (zero padding). */
ORACLE_API void oracle_adjoint_f64(int W, int H, int D, int S, const float *w, const int *off, const int *rows,
                                   const int *cols, const float *var, const uint8_t *smap, const double *g,
                                   double *grad) {
    int nk = D * S;
    int *begin = (int *)malloc(sizeof(int) * (nk + 1));
    tap_t *taps = build_taps(w, off, rows, cols, nk, begin);
    size_t npx = (size_t)W * H;
    double *alpha = (double *)malloc(sizeof(double) * D);
    memset(grad, 0, sizeof(double) * npx);
    for (int py = 0; py < H; py++)
        for (int px = 0; px < W; px++) {
            size_t p = (size_t)py * W + px;
            frozen_alpha(smap, npx, D, S, var, p, alpha);
            for (int d = 0; d < D; d++) {
                int k = d * S + smap[(size_t)d * npx + p];
                double c = g[p] * alpha[d];
                for (int t = begin[k]; t < begin[k + 1]; t++) {
                    int iy = py + taps[t].dy, ix = px + taps[t].dx;
                    if (iy >= 0 && iy < H && ix >= 0 && ix < W) grad[(size_t)iy * W + ix] += c * taps[t].w;
                }
            }
        }
    free(alpha);
    free(taps);
    free(begin);
}

/* Frozen-selection loss restricted to the pixels a change at q can reach:
 *   L_q(x) = sum_{p : |p - q| <= R} g[p] * sum_d alpha_d(p) * e_{d,s*(d,p)}(p; x),   R = max radius. */
static double frozen_local_loss(const float *x, double xq, size_t q, int W, int H, int D, int S, const tap_t *taps,
                                const int *begin, int R, const float *var, const uint8_t *smap, const double *g) {
    size_t npx = (size_t)W * H;
    int qy = (int)(q / W), qx = (int)(q % W);
    double *alpha = (double *)malloc(sizeof(double) * D);
    double L = 0.0;
    for (int py = qy - R; py <= qy + R; py++) {
        if (py < 0 || py >= H) continue;
        for (int px = qx - R; px <= qx + R; px++) {
            if (px < 0 || px >= W) continue;
            size_t p = (size_t)py * W + px;
            frozen_alpha(smap, npx, D, S, var, p, alpha);
            double o = 0.0;
            for (int d = 0; d < D; d++) {
                int k = d * S + smap[(size_t)d * npx + p];
                double e = 0.0;
                for (int t = begin[k]; t < begin[k + 1]; t++) {
                    int iy = py + taps[t].dy, ix = px + taps[t].dx;
                    if (iy >= 0 && iy < H && ix >= 0 && ix < W) {
                        size_t i = (size_t)iy * W + ix;
                        e += (double)taps[t].w * (i == q ? xq : (double)x[i]);
                    }
                }
                o += alpha[d] * e;
            }
            L += g[p] * o;
        }
    }
    free(alpha);
    return L;
}

/* Central finite differences (L(x + eps e_q) - L(x - eps e_q)) / (2 eps) of the frozen-selection
 * loss sum_p g[p] * out[p], at the n pixels q[i], in double. */
ORACLE_API void oracle_fd_grad_f64(const float *x, int W, int H, int D, int S, const float *w, const int *off,
                                   const int *rows, const int *cols, const float *var, const uint8_t *smap,
                                   const double *g, const long *q, int n, double eps, double *fd) {
    int nk = D * S;
    int *begin = (int *)malloc(sizeof(int) * (nk + 1));
    tap_t *taps = build_taps(w, off, rows, cols, nk, begin);
    int R = 0;
    for (int k = 0; k < nk; k++) {
        if (rows[k] / 2 > R) R = rows[k] / 2;
        if (cols[k] / 2 > R) R = cols[k] / 2;
    }
    for (int i = 0; i < n; i++) {
        double x0 = (double)x[q[i]];
        double Lp = frozen_local_loss(x, x0 + eps, (size_t)q[i], W, H, D, S, taps, begin, R, var, smap, g);
        double Lm = frozen_local_loss(x, x0 - eps, (size_t)q[i], W, H, D, S, taps, begin, R, var, smap, g);
        fd[i] = (Lp - Lm) / (2.0 * eps);
    }
    free(taps);
    free(begin);
}
