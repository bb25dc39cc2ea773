/*
 * polycrystal.c -- oracle-side generator of the synthetic polycrystals (see
 * polycrystal.h for the recipe).  TEST-ORACLE INFRASTRUCTURE.
 *
 * Compile with -ffp-contract=off: the orientations must come out bit for bit
 * as the product's generator makes them, whatever -march the caller uses.
 */
#include "polycrystal.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t s;
} splitmix64;

static uint64_t sm_next(splitmix64 *r) {
  r->s += 0x9E3779B97F4A7C15ull;
  uint64_t z = r->s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double sm_u01(splitmix64 *r) { return (double)(sm_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* active rotation matrix of the unit quaternion (w, x, y, z), row-major */
static void quat_rotation(double w, double x, double y, double z, double *R) {
  R[0] = 1 - 2 * (y * y + z * z);
  R[1] = 2 * (x * y - w * z);
  R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z);
  R[4] = 1 - 2 * (x * x + z * z);
  R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y);
  R[7] = 2 * (y * z + w * x);
  R[8] = 1 - 2 * (x * x + y * y);
}

static double lesser(double a, double b) { return (b < a) ? b : a; }

/* squared minimum-image distance of (x, y, z) to seed p on an n-periodic box */
static double periodic_d2(double x, double y, double z, const double *p, int nx, int ny, int nz) {
  double dx = fabs(x - p[0]);
  dx = lesser(dx, nx - dx);
  double dy = fabs(y - p[1]);
  dy = lesser(dy, ny - dy);
  double dz = fabs(z - p[2]);
  dz = lesser(dz, nz - dz);
  return dx * dx + dy * dy + dz * dz;
}

typedef struct {
  int nx, ny, nz, grains;
  int nb[3];        /* buckets per axis */
  double bw[3];     /* bucket width per axis */
  int *start, *idx; /* seeds of bucket b: idx[start[b] .. start[b+1]), ascending */
  const double *pts, *rot;
  double *R;
  int32_t *grain;
  int x0, x1;
} gen_job;

static int bucket_of(const gen_job *j, int a, double v) {
  int c = (int)floor(v / j->bw[a]);
  return c < j->nb[a] - 1 ? c : j->nb[a] - 1;
}

static int wrap(int c, int n) { return ((c % n) + n) % n; }

static void *gen_rows(void *arg) {
  const gen_job *j = (const gen_job *)arg;
  const int nmax = j->nb[0] > j->nb[1] ? (j->nb[0] > j->nb[2] ? j->nb[0] : j->nb[2])
                                       : (j->nb[1] > j->nb[2] ? j->nb[1] : j->nb[2]);
  for (int x = j->x0; x < j->x1; ++x)
    for (int y = 0; y < j->ny; ++y)
      for (int z = 0; z < j->nz; ++z) {
        const double pos[3] = {(double)x, (double)y, (double)z};
        int home[3];
        for (int a = 0; a < 3; ++a) home[a] = bucket_of(j, a, pos[a]);
        double best = INFINITY;
        int bi = 0x7fffffff;
        for (int r = 0; r <= nmax; ++r) {
          /* the shell of buckets at Chebyshev distance r from the home bucket */
          for (int dx = -r; dx <= r; ++dx)
            for (int dy = -r; dy <= r; ++dy)
              for (int dz = -r; dz <= r; ++dz) {
                int ax = abs(dx), ay = abs(dy), az = abs(dz);
                int m = ax > ay ? ax : ay;
                m = m > az ? m : az;
                if (m != r) continue;
                const int b = (wrap(home[0] + dx, j->nb[0]) * j->nb[1] +
                               wrap(home[1] + dy, j->nb[1])) * j->nb[2] +
                              wrap(home[2] + dz, j->nb[2]);
                for (int k = j->start[b]; k < j->start[b + 1]; ++k) {
                  const int g = j->idx[k];
                  const double d2 =
                      periodic_d2(pos[0], pos[1], pos[2], j->pts + 3 * (size_t)g, j->nx, j->ny, j->nz);
                  if (d2 < best || (d2 == best && g < bi)) {
                    best = d2;
                    bi = g;
                  }
                }
              }
          /* a seed outside the searched block is at least this far away
             along some axis the block does not cover */
          double lb = INFINITY;
          int covered = 1;
          for (int a = 0; a < 3; ++a) {
            if (2 * r + 1 >= j->nb[a]) continue;
            covered = 0;
            const double lo = (home[a] - r) * j->bw[a], hi = (home[a] + r + 1) * j->bw[a];
            lb = lesser(lb, lesser(pos[a] - lo, hi - pos[a]));
          }
          if (covered || best < lb * lb) break;
        }
        const size_t v = ((size_t)x * j->ny + y) * j->nz + z;
        memcpy(j->R + 9 * v, j->rot + 9 * (size_t)bi, sizeof(double) * 9);
        if (j->grain) j->grain[v] = bi;
      }
  return NULL;
}

int oracle_polycrystal(int nx, int ny, int nz, int grains, uint64_t seed, int threads,
                       double *R_out, int32_t *grain_out) {
  if (nx < 1 || ny < 1 || nz < 1 || grains < 1 || !R_out) return 1;
  double *pts = (double *)malloc(sizeof(double) * 3 * (size_t)grains);
  double *rot = (double *)malloc(sizeof(double) * 9 * (size_t)grains);
  if (!pts || !rot) return 2;
  splitmix64 rng = {seed};
  const double two_pi = 6.283185307179586476925286766559;
  for (int g = 0; g < grains; ++g) {
    pts[3 * g + 0] = sm_u01(&rng) * nx;
    pts[3 * g + 1] = sm_u01(&rng) * ny;
    pts[3 * g + 2] = sm_u01(&rng) * nz;
    const double u1 = sm_u01(&rng), u2 = sm_u01(&rng), u3 = sm_u01(&rng);
    const double a = sqrt(1.0 - u1), b = sqrt(u1);
    const double qx = a * sin(two_pi * u2), qy = a * cos(two_pi * u2);
    const double qz = b * sin(two_pi * u3), qw = b * cos(two_pi * u3);
    quat_rotation(qw, qx, qy, qz, rot + 9 * (size_t)g);
  }
  gen_job base;
  memset(&base, 0, sizeof(base));
  base.nx = nx;
  base.ny = ny;
  base.nz = nz;
  base.grains = grains;
  const int dims[3] = {nx, ny, nz};
  int per = (int)floor(cbrt((double)grains));
  if (per < 1) per = 1;
  for (int a = 0; a < 3; ++a) {
    base.nb[a] = per < dims[a] ? per : dims[a];
    base.bw[a] = (double)dims[a] / base.nb[a];
  }
  const int nbuckets = base.nb[0] * base.nb[1] * base.nb[2];
  int *count = (int *)calloc((size_t)nbuckets + 1, sizeof(int));
  int *start = (int *)calloc((size_t)nbuckets + 1, sizeof(int));
  int *idx = (int *)malloc(sizeof(int) * (size_t)grains);
  int *home = (int *)malloc(sizeof(int) * (size_t)grains);
  for (int g = 0; g < grains; ++g) {
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = bucket_of(&base, a, pts[3 * g + a]);
    home[g] = (c[0] * base.nb[1] + c[1]) * base.nb[2] + c[2];
    count[home[g]]++;
  }
  for (int b = 0; b < nbuckets; ++b) start[b + 1] = start[b] + count[b];
  memset(count, 0, sizeof(int) * (size_t)nbuckets);
  for (int g = 0; g < grains; ++g) idx[start[home[g]] + count[home[g]]++] = g;
  base.start = start;
  base.idx = idx;
  base.pts = pts;
  base.rot = rot;
  base.R = R_out;
  base.grain = grain_out;
  if (threads < 1) threads = 1;
  if (threads > nx) threads = nx;
  gen_job *jobs = (gen_job *)malloc(sizeof(gen_job) * (size_t)threads);
  pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int t = 0; t < threads; ++t) {
    jobs[t] = base;
    jobs[t].x0 = (int)((long long)nx * t / threads);
    jobs[t].x1 = (int)((long long)nx * (t + 1) / threads);
    if (t > 0) pthread_create(&tid[t], NULL, gen_rows, &jobs[t]);
  }
  gen_rows(&jobs[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
  free(jobs);
  free(tid);
  free(count);
  free(start);
  free(idx);
  free(home);
  free(pts);
  free(rot);
  return 0;
}
