/*
 * dft.c -- see dft.h.  Test-oracle code only.
 */
#include "dft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAX_FACTORS 64

struct oracle_dft1d {
  size_t n;
  int sign;
  int nfac;
  size_t fac[MAX_FACTORS];
  oracle_cplx *tw; /* tw[j] = exp(sign * 2 pi i j / n), j in [0, n) */
};

static void factorize(size_t n, size_t *fac, int *nfac) {
  int k = 0;
  /* radix-4 first (fewer combine stages), then 2, 3, 5, then any prime */
  while (n % 4 == 0 && n > 4) { fac[k++] = 4; n /= 4; }
  while (n % 2 == 0) { fac[k++] = 2; n /= 2; }
  while (n % 3 == 0) { fac[k++] = 3; n /= 3; }
  while (n % 5 == 0) { fac[k++] = 5; n /= 5; }
  for (size_t p = 7; n > 1; p += 2) {
    while (n % p == 0) { fac[k++] = p; n /= p; }
  }
  *nfac = k;
}

oracle_dft1d *oracle_dft1d_plan(size_t n, int sign) {
  oracle_dft1d *p = (oracle_dft1d *)calloc(1, sizeof(*p));
  if (!p) return NULL;
  p->n = n;
  p->sign = sign;
  if (n > 1) factorize(n, p->fac, &p->nfac);
  p->tw = (oracle_cplx *)malloc(sizeof(oracle_cplx) * (n ? n : 1));
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (size_t j = 0; j < n; ++j) {
    long double a = two_pi * (long double)j / (long double)n;
    p->tw[j].re = (double)cosl(a);
    p->tw[j].im = (double)(sign * sinl(a));
  }
  return p;
}

void oracle_dft1d_free(oracle_dft1d *p) {
  if (!p) return;
  free(p->tw);
  free(p);
}

static inline oracle_cplx cmul(oracle_cplx a, oracle_cplx b) {
  oracle_cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

/* Recursive DIT: out[0..n) = DFT_n of in[0], in[is], ..., in[(n-1) is].
 * Twiddle W_n^e = tw[(e mod n) * tws], where tw covers the full length. */
static void dit(const oracle_dft1d *P, const oracle_cplx *in, size_t is, oracle_cplx *out,
                size_t n, const size_t *fac, size_t tws) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  const size_t p = fac[0];
  const size_t m = n / p;
  for (size_t q = 0; q < p; ++q) dit(P, in + q * is, is * p, out + q * m, m, fac + 1, tws * p);

  oracle_cplx t[MAX_FACTORS > 64 ? MAX_FACTORS : 64];
  oracle_cplx *tbuf = t;
  oracle_cplx *heap = NULL;
  if (p > 64) {
    heap = (oracle_cplx *)malloc(sizeof(oracle_cplx) * p);
    tbuf = heap;
  }
  for (size_t k = 0; k < m; ++k) {
    for (size_t q = 0; q < p; ++q) {
      oracle_cplx y = out[q * m + k];
      size_t e = (q * k) % n;
      tbuf[q] = q == 0 ? y : cmul(y, P->tw[e * tws]);
    }
    if (p == 2) {
      oracle_cplx a = tbuf[0], b = tbuf[1];
      out[k].re = a.re + b.re; out[k].im = a.im + b.im;
      out[k + m].re = a.re - b.re; out[k + m].im = a.im - b.im;
    } else if (p == 4) {
      /* W_4 = exp(sign*i*pi/2) = sign*i */
      const double s = (double)P->sign;
      oracle_cplx a0 = tbuf[0], a1 = tbuf[1], a2 = tbuf[2], a3 = tbuf[3];
      oracle_cplx u0 = {a0.re + a2.re, a0.im + a2.im};
      oracle_cplx u1 = {a0.re - a2.re, a0.im - a2.im};
      oracle_cplx u2 = {a1.re + a3.re, a1.im + a3.im};
      oracle_cplx u3 = {a1.re - a3.re, a1.im - a3.im};
      /* (sign*i) * u3 */
      oracle_cplx v3 = {-s * u3.im, s * u3.re};
      out[k].re = u0.re + u2.re;           out[k].im = u0.im + u2.im;
      out[k + m].re = u1.re + v3.re;       out[k + m].im = u1.im + v3.im;
      out[k + 2 * m].re = u0.re - u2.re;   out[k + 2 * m].im = u0.im - u2.im;
      out[k + 3 * m].re = u1.re - v3.re;   out[k + 3 * m].im = u1.im - v3.im;
    } else {
      /* direct p-point DFT with W_p^{qs} = W_n^{qs m} */
      for (size_t s = 0; s < p; ++s) {
        oracle_cplx acc = tbuf[0];
        for (size_t q = 1; q < p; ++q) {
          size_t e = ((q * s) % p) * m;
          oracle_cplx w = P->tw[e * tws];
          acc.re += tbuf[q].re * w.re - tbuf[q].im * w.im;
          acc.im += tbuf[q].re * w.im + tbuf[q].im * w.re;
        }
        out[k + s * m] = acc;
      }
    }
  }
  free(heap);
}

void oracle_dft1d_exec(const oracle_dft1d *p, const oracle_cplx *in, size_t is, oracle_cplx *out,
                       size_t os) {
  if (p->n == 0) return;
  if (os == 1) {
    dit(p, in, is, out, p->n, p->fac, 1);
    return;
  }
  oracle_cplx *tmp = (oracle_cplx *)malloc(sizeof(oracle_cplx) * p->n);
  dit(p, in, is, tmp, p->n, p->fac, 1);
  for (size_t k = 0; k < p->n; ++k) out[k * os] = tmp[k];
  free(tmp);
}

void oracle_dft3d_inplace(oracle_cplx *data, size_t n0, size_t n1, size_t n2, int sign) {
  size_t dims[3] = {n0, n1, n2};
  size_t strides[3] = {n1 * n2, n2, 1};
  size_t nmax = n0 > n1 ? n0 : n1;
  if (n2 > nmax) nmax = n2;
  oracle_cplx *line = (oracle_cplx *)malloc(sizeof(oracle_cplx) * nmax);
  oracle_cplx *res = (oracle_cplx *)malloc(sizeof(oracle_cplx) * nmax);
  for (int ax = 2; ax >= 0; --ax) {
    size_t n = dims[ax];
    if (n <= 1) continue;
    oracle_dft1d *p = oracle_dft1d_plan(n, sign);
    size_t st = strides[ax];
    /* iterate over all lines along axis ax */
    size_t total = n0 * n1 * n2;
    for (size_t base = 0; base < total; ++base) {
      /* base is a line start iff its coordinate along ax is 0 */
      size_t coord = (base / st) % n;
      if (coord != 0) continue;
      for (size_t j = 0; j < n; ++j) line[j] = data[base + j * st];
      dit(p, line, 1, res, n, p->fac, 1);
      for (size_t j = 0; j < n; ++j) data[base + j * st] = res[j];
    }
    oracle_dft1d_free(p);
  }
  free(line);
  free(res);
}
