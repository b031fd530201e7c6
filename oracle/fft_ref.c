/*
 * CPU DFT for the oracle (test infrastructure only; see fft_ref.h).
 */
#include "fft_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

int ora_fft_init(ora_fft *p, int len) {
    memset(p, 0, sizeof(*p));
    if (len < 1) return -1;
    p->len  = len;
    p->pow2 = is_pow2(len);
    p->cs   = (double *)malloc(sizeof(double) * (size_t)len);
    p->sn   = (double *)malloc(sizeof(double) * (size_t)len);
    p->work = (double *)malloc(sizeof(double) * 4 * (size_t)len);
    if (!p->cs || !p->sn || !p->work) { ora_fft_free(p); return -1; }
    for (int t = 0; t < len; t++) {
        /* angle reduced to the first period before evaluation */
        double a = 2.0 * M_PI * (double)t / (double)len;
        p->cs[t] = cos(a);
        p->sn[t] = sin(a);
    }
    if (p->pow2) {
        int bits = 0;
        while ((1 << bits) < len) bits++;
        p->rev = (int *)malloc(sizeof(int) * (size_t)len);
        if (!p->rev) { ora_fft_free(p); return -1; }
        for (int i = 0; i < len; i++) {
            int r = 0;
            for (int b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);
            p->rev[i] = r;
        }
    }
    return 0;
}

void ora_fft_free(ora_fft *p) {
    free(p->cs);
    free(p->sn);
    free(p->rev);
    free(p->work);
    memset(p, 0, sizeof(*p));
}

static void fft_radix2(const ora_fft *p, double *d) {
    const int n = p->len;
    for (int i = 0; i < n; i++) {
        int r = p->rev[i];
        if (r > i) {
            double tr = d[2 * i], ti = d[2 * i + 1];
            d[2 * i] = d[2 * r];
            d[2 * i + 1] = d[2 * r + 1];
            d[2 * r] = tr;
            d[2 * r + 1] = ti;
        }
    }
    for (int half = 1; half < n; half <<= 1) {
        const int step = n / (2 * half); /* twiddle index stride */
        for (int base = 0; base < n; base += 2 * half) {
            for (int q = 0; q < half; q++) {
                /* w = exp(-2 pi i q / (2 half)) = cos - i sin */
                double wr = p->cs[q * step], wi = -p->sn[q * step];
                double *a = d + 2 * (base + q);
                double *b = d + 2 * (base + q + half);
                double br = b[0] * wr - b[1] * wi;
                double bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br;
                b[1] = a[1] - bi;
                a[0] = a[0] + br;
                a[1] = a[1] + bi;
            }
        }
    }
}

static void dft_direct(const ora_fft *p, double *d) {
    const int n = p->len;
    double *w = p->work + 2 * (size_t)n;
    for (int k = 0; k < n; k++) {
        double sr = 0.0, si = 0.0;
        long   t  = 0; /* (k*j) mod n, advanced incrementally */
        for (int j = 0; j < n; j++) {
            double c = p->cs[t], s = -p->sn[t];
            sr += d[2 * j] * c - d[2 * j + 1] * s;
            si += d[2 * j] * s + d[2 * j + 1] * c;
            t += k;
            if (t >= n) t -= n;
        }
        w[2 * k]     = sr;
        w[2 * k + 1] = si;
    }
    memcpy(d, w, sizeof(double) * 2 * (size_t)n);
}

void ora_fft_c2c(const ora_fft *p, double *data) {
    if (p->pow2) fft_radix2(p, data);
    else dft_direct(p, data);
}

void ora_fft_r2c(const ora_fft *p, const double *in, double *out) {
    const int n = p->len;
    /* first half of `work` stages the data; dft_direct uses the second half */
    double *tmp = p->work;
    for (int i = 0; i < n; i++) {
        tmp[2 * i]     = in[i];
        tmp[2 * i + 1] = 0.0;
    }
    ora_fft_c2c(p, tmp);
    memcpy(out, tmp, sizeof(double) * 2 * (size_t)(n / 2 + 1));
}
