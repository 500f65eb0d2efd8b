/*
 * FP64 CPU oracle for the apoCHARMM force-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the test-suite, the smoke check and the
 * CPU-baseline leg of the benchmark load this library, as the checker and as
 * the timed CPU reference.  The product (libapocharmm_c.so) never links it.
 *
 * Every routine restates, in double precision, the algorithm the reference
 * engine runs on the GPU (citations are paths inside the reference project):
 *
 *   direct space   src/CudaDirectForceKernels.cu:465-489 (erfc-Ewald),
 *                  :263-286 (VDW_VFSW), setup constants
 *                  src/CudaPMEDirectForce.cu:275-391, pair loop
 *                  include/CudaDirectForce_util.h:134-248 (r2 < roff2 test,
 *                  gradient = (r dU/dr)/r^2 * (xi - xj)).
 *   1-4 / excl.    src/CudaDirectForceKernels.cu:643-870 (in14 with
 *                  e14fac = 1: LJ14 + qq erfc/r, ex14: qq (erfc-1)/r, both
 *                  with ishift 13, i.e. raw coordinate differences).
 *   reciprocal     include/cuda_pme_spread.h:64-141 (grid anchoring
 *                  w = x/L + 2, fr = n (w - (floor(w+0.5)-0.5)), points
 *                  floor(fr)+0..p-1), src/CudaPMERecip.cu:438-470 (B-spline
 *                  recursion), :674-929 (influence function, energy with the
 *                  conjugate term for k1 >= 1, virial), :2656-2758 (moduli),
 *                  include/cuda_pme_gather.h:140-320 (gradient).
 *   self energy    include/cuda_pme_selfe.h:337-375.
 *   bonded         src/CudaBondedForce.cu:85-760.
 *
 * Units: kcal/mol, Angstrom, e.  All outputs are GRADIENTS (dU/dx), the
 * reference's force-buffer convention (src/CudaLeapFrogIntegrator.cu:33).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CCELEC 332.0716
#define PI 3.14159265358979323846

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

int or_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* pair functions                                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  double roff, ron, roff2, ron2, kappa;
  double k6, k12, dv6, dv12, roffinv3, roffinv6;
} nb_setup;

static void nb_setup_init(nb_setup *s, double kappa, double roff, double ron) {
  s->roff = roff;
  s->ron = ron;
  s->roff2 = roff * roff;
  s->ron2 = ron * ron;
  s->kappa = kappa;
  double roff3 = roff * roff * roff, ron3 = ron * ron * ron;
  double roff6 = roff3 * roff3, ron6 = ron3 * ron3;
  s->roffinv3 = 1.0 / roff3;
  s->roffinv6 = 1.0 / roff6;
  if (ron < roff) {
    s->k6 = roff3 / (roff3 - ron3);
    s->k12 = roff6 / (roff6 - ron6);
    s->dv6 = -1.0 / (ron3 * roff3);
    s->dv12 = -1.0 / (ron6 * roff6);
  } else {
    s->k6 = 1.0;
    s->k12 = 1.0;
    s->dv6 = -1.0 / roff6;
    s->dv12 = -1.0 / (roff6 * roff6);
  }
}

/* CHARMM force-switched LJ (VDW_VFSW).  c6, c12 are the raw pair
 * coefficients (c6 = 2 eps rmin^6, c12 = eps rmin^12).  Returns r dU/dr. */
static double vfsw(const nb_setup *s, double r2, double c6, double c12,
                   double *e) {
  double rinv2 = 1.0 / r2;
  double rinv3 = sqrt(rinv2) * rinv2;
  double rinv6 = rinv3 * rinv3;
  int sw = r2 > s->ron2;
  double A6 = sw ? s->k6 : 1.0, B6 = sw ? s->roffinv3 : 0.0;
  double A12 = sw ? s->k12 : 1.0, B12 = sw ? s->roffinv6 : 0.0;
  double C6 = sw ? 0.0 : s->dv6, C12 = sw ? 0.0 : s->dv12;
  double t6 = rinv3 - B6, t12 = rinv6 - B12;
  *e = c12 * (A12 * t12 * t12 + C12) - c6 * (A6 * t6 * t6 + C6);
  return 6.0 * c6 * A6 * t6 * rinv3 - 12.0 * c12 * A12 * t12 * rinv6;
}

/* qq * (erfc(kr) + fac) / r; returns r dU/dr. */
static double ewald_pair(double kappa, double r, double qq, double fac,
                         double *e) {
  double erfcv = erfc(kappa * r);
  double expv = exp(-kappa * kappa * r * r);
  double v = qq * (erfcv + fac) / r;
  *e = v;
  return -qq * (2.0 / sqrt(PI)) * kappa * expv - v;
}

/* ------------------------------------------------------------------------ */
/* direct space                                                             */
/* ------------------------------------------------------------------------ */

static int is_excluded(int i, int j, const int *ptr, const int *idx) {
  int lo = ptr[i], hi = ptr[i + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (idx[mid] == j) return 1;
    if (idx[mid] < j) lo = mid + 1;
    else hi = mid;
  }
  return 0;
}

/*
 * Real-space erfc-Ewald + VFSW LJ over all minimum-image pairs with
 * r < roff that are not topologically excluded (1-2, 1-3, 1-4).
 * excl_ptr/excl_idx: symmetric CSR, partners sorted ascending.
 * c6c12: full ntype x ntype x 2 table of raw coefficients.
 * Each atom sums over all its partners (pairs visited twice, energy halved),
 * so the result does not depend on thread scheduling.
 */
int or_direct(int n, const double *xyz, const double *q, const int *type,
              int ntype, const double *c6c12, const int *excl_ptr,
              const int *excl_idx, const double *box, double kappa,
              double roff, double ron, double *grad, double *e_elec,
              double *e_vdw, double *vir9, int nthreads) {
  nb_setup s;
  nb_setup_init(&s, kappa, roff, ron);
  set_threads(nthreads);
  int nc[3];
  for (int d = 0; d < 3; d++) {
    nc[d] = (int)floor(box[d] / roff);
    if (nc[d] < 3) nc[d] = 1;
  }
  int ncell = nc[0] * nc[1] * nc[2];
  int *head = (int *)malloc(sizeof(int) * ncell);
  int *next = (int *)malloc(sizeof(int) * n);
  int *cellof = (int *)malloc(sizeof(int) * n);
  if (!head || !next || !cellof) return -1;
  for (int c = 0; c < ncell; c++) head[c] = -1;
  for (int i = 0; i < n; i++) {
    int ci[3];
    for (int d = 0; d < 3; d++) {
      double f = xyz[3 * i + d] / box[d] + 0.5;
      f -= floor(f);
      ci[d] = (int)(f * nc[d]);
      if (ci[d] >= nc[d]) ci[d] = nc[d] - 1;
    }
    int c = ci[0] + nc[0] * (ci[1] + nc[1] * ci[2]);
    cellof[i] = c;
  }
  for (int i = n - 1; i >= 0; i--) {
    next[i] = head[cellof[i]];
    head[cellof[i]] = i;
  }
  double ee = 0.0, ev = 0.0;
  double w0 = 0, w1 = 0, w2 = 0, w3 = 0, w4 = 0, w5 = 0, w6 = 0, w7 = 0, w8 = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : ee, ev, w0, w1, w2, w3, w4, w5, w6, w7, w8)
  for (int i = 0; i < n; i++) {
    int c = cellof[i];
    int cx = c % nc[0], cy = (c / nc[0]) % nc[1], cz = c / (nc[0] * nc[1]);
    double gx = 0, gy = 0, gz = 0;
    int rx = nc[0] >= 3 ? 1 : 0, ry = nc[1] >= 3 ? 1 : 0,
        rz = nc[2] >= 3 ? 1 : 0;
    for (int dz = -rz; dz <= rz; dz++)
      for (int dy = -ry; dy <= ry; dy++)
        for (int dx = -rx; dx <= rx; dx++) {
          int ox = (cx + dx + nc[0]) % nc[0], oy = (cy + dy + nc[1]) % nc[1],
              oz = (cz + dz + nc[2]) % nc[2];
          for (int j = head[ox + nc[0] * (oy + nc[1] * oz)]; j >= 0;
               j = next[j]) {
            if (j == i) continue;
            double d[3];
            for (int k = 0; k < 3; k++) {
              d[k] = xyz[3 * i + k] - xyz[3 * j + k];
              d[k] -= box[k] * round(d[k] / box[k]);
            }
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 >= s.roff2) continue;
            if (is_excluded(i, j, excl_ptr, excl_idx)) continue;
            double r = sqrt(r2);
            double eel, evd;
            double fr = ewald_pair(kappa, r, CCELEC * q[i] * q[j], 0.0, &eel);
            int ti = type[i], tj = type[j];
            double c6 = c6c12[2 * (ti * ntype + tj)],
                   c12 = c6c12[2 * (ti * ntype + tj) + 1];
            fr += vfsw(&s, r2, c6, c12, &evd);
            ee += 0.5 * eel;
            ev += 0.5 * evd;
            double f = fr / r2;
            gx += f * d[0];
            gy += f * d[1];
            gz += f * d[2];
            /* virial -sum over pairs of d (x) gradient_i; pairs visited twice */
            double h = -0.5 * f;
            w0 += h * d[0] * d[0]; w1 += h * d[0] * d[1]; w2 += h * d[0] * d[2];
            w3 += h * d[1] * d[0]; w4 += h * d[1] * d[1]; w5 += h * d[1] * d[2];
            w6 += h * d[2] * d[0]; w7 += h * d[2] * d[1]; w8 += h * d[2] * d[2];
          }
        }
    grad[3 * i + 0] += gx;
    grad[3 * i + 1] += gy;
    grad[3 * i + 2] += gz;
  }
  free(head);
  free(next);
  free(cellof);
  *e_elec = ee;
  *e_vdw = ev;
  if (vir9) {
    vir9[0] += w0; vir9[1] += w1; vir9[2] += w2;
    vir9[3] += w3; vir9[4] += w4; vir9[5] += w5;
    vir9[6] += w6; vir9[7] += w7; vir9[8] += w8;
  }
  return 0;
}

/* 1-4 inclusions (LJ14 + qq erfc/r; energies to vdw / elec) and 1-2/1-3
 * exclusion corrections (qq (erfc-1)/r; energy to ewex).  Raw coordinate
 * differences (ishift 13), no cutoff test, as in the reference. */
int or_14(int nin, const int *in14, int nex, const int *ex14, const double *xyz,
          const double *q, const int *type, int ntype, const double *c6c12_14,
          double kappa, double roff, double ron, double *grad, double *e_elec,
          double *e_vdw, double *e_ewex) {
  nb_setup s;
  nb_setup_init(&s, kappa, roff, ron);
  double ee = 0, ev = 0, ex = 0;
  for (int p = 0; p < nin + nex; p++) {
    int incl = p < nin;
    int i = incl ? in14[2 * p] : ex14[2 * (p - nin)];
    int j = incl ? in14[2 * p + 1] : ex14[2 * (p - nin) + 1];
    double d[3];
    for (int k = 0; k < 3; k++) d[k] = xyz[3 * i + k] - xyz[3 * j + k];
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double r = sqrt(r2);
    double qq = CCELEC * q[i] * q[j];
    double e1, e2, fr;
    if (incl) {
      fr = ewald_pair(kappa, r, qq, 0.0, &e1);
      int ti = type[i], tj = type[j];
      fr += vfsw(&s, r2, c6c12_14[2 * (ti * ntype + tj)],
                 c6c12_14[2 * (ti * ntype + tj) + 1], &e2);
      ee += e1;
      ev += e2;
    } else {
      fr = ewald_pair(kappa, r, qq, -1.0, &e1);
      ex += e1;
    }
    double f = fr / r2;
    for (int k = 0; k < 3; k++) {
      grad[3 * i + k] += f * d[k];
      grad[3 * j + k] -= f * d[k];
    }
  }
  *e_elec = ee;
  *e_vdw = ev;
  *e_ewex = ex;
  return 0;
}

double or_self_energy(int n, const double *q, double kappa) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += q[i] * q[i];
  return -kappa * CCELEC / sqrt(PI) * s;
}

/* ------------------------------------------------------------------------ */
/* FFT (complex, any length; mixed radix by recursion on the smallest prime) */
/* ------------------------------------------------------------------------ */

static void fft_rec(int n, const double *in, int istride, double *out,
                    double sign, double *scratch) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  int p = 2;
  while (p * p <= n && n % p) p++;
  if (n % p) p = n; /* prime length: direct DFT */
  int m = n / p;
  /* sub-transforms of the decimated sequences */
  for (int r = 0; r < p; r++)
    fft_rec(m, in + 2 * r * istride, istride * p, scratch + 2 * r * m, sign,
            out);
  for (int k = 0; k < m; k++) {
    for (int s = 0; s < p; s++) {
      double re = 0, im = 0;
      for (int r = 0; r < p; r++) {
        double ang = sign * 2.0 * PI * (double)r * (double)(k + s * m) / n;
        double c = cos(ang), sn = sin(ang);
        double xr = scratch[2 * (r * m + k)], xi = scratch[2 * (r * m + k) + 1];
        re += xr * c - xi * sn;
        im += xr * sn + xi * c;
      }
      out[2 * (k + s * m)] = re;
      out[2 * (k + s * m) + 1] = im;
    }
  }
}

/* in-place complex FFT of n points with element stride `stride` (in complex
 * units) inside `data`; sign -1 forward, +1 backward, unnormalised. */
static void fft_line(double *data, int n, int stride, double sign, double *buf) {
  double *a = buf, *b = buf + 2 * n, *c = buf + 4 * n;
  for (int k = 0; k < n; k++) {
    a[2 * k] = data[2 * k * stride];
    a[2 * k + 1] = data[2 * k * stride + 1];
  }
  fft_rec(n, a, 1, b, sign, c);
  for (int k = 0; k < n; k++) {
    data[2 * k * stride] = b[2 * k];
    data[2 * k * stride + 1] = b[2 * k + 1];
  }
}

/* full complex 3D FFT of a (nx, ny, nz) grid, x fastest */
static void fft3d(double *g, int nx, int ny, int nz, double sign) {
  int nmax = nx > ny ? nx : ny;
  if (nz > nmax) nmax = nz;
#pragma omp parallel
  {
    /* fft_rec uses up to ~n*(1 + 1/2 + ...) scratch per level */
    double *buf = (double *)malloc(sizeof(double) * 2 * 8 * nmax);
#pragma omp for
    for (int l = 0; l < ny * nz; l++) fft_line(g + 2 * (l * nx), nx, 1, sign, buf);
#pragma omp for
    for (int l = 0; l < nx * nz; l++) {
      int x = l % nx, z = l / nx;
      fft_line(g + 2 * (x + nx * ny * z), ny, nx, sign, buf);
    }
#pragma omp for
    for (int l = 0; l < nx * ny; l++) fft_line(g + 2 * l, nz, nx * ny, sign, buf);
    free(buf);
  }
}

/* ------------------------------------------------------------------------ */
/* PME                                                                       */
/* ------------------------------------------------------------------------ */

/* B-spline weights and derivatives, reference src/CudaPMERecip.cu:438-470 */
static void bspline(double w, int order, double *th, double *dth) {
  th[order - 1] = 0.0;
  th[1] = w;
  th[0] = 1.0 - w;
  for (int k = 3; k <= order - 1; k++) {
    double div = 1.0 / (double)(k - 1);
    th[k - 1] = div * w * th[k - 2];
    for (int j = 1; j <= k - 2; j++)
      th[k - j - 1] = div * ((w + j) * th[k - j - 2] + (k - j - w) * th[k - j - 1]);
    th[0] = div * (1.0 - w) * th[0];
  }
  dth[0] = -th[0];
  for (int j = 1; j < order; j++) dth[j] = th[j - 1] - th[j];
  double div = 1.0 / (double)(order - 1);
  th[order - 1] = div * w * th[order - 2];
  for (int j = 1; j <= order - 2; j++)
    th[order - j - 1] =
        div * ((w + j) * th[order - j - 2] + (order - j - w) * th[order - j - 1]);
  th[0] = div * (1.0 - w) * th[0];
}

/* 1/|b(k)|^2 as in the reference's dftmod (src/CudaPMERecip.cu:2656-2678) */
static void bspline_moduli(int nfft, int order, double *prefac) {
  double th[16], dth[16];
  double *arr = (double *)calloc(nfft + order + 2, sizeof(double));
  bspline(0.0, order, th, dth);
  for (int i = 2; i <= order + 1; i++) arr[i - 1] = th[i - 2];
  for (int k = 0; k < nfft; k++) {
    double s1 = 0, s2 = 0;
    for (int j = 0; j < nfft - 1; j++) {
      double a = 2.0 * PI * k * j / nfft;
      s1 += arr[j] * cos(a);
      s2 += arr[j] * sin(a);
    }
    prefac[k] = s1 * s1 + s2 * s2;
  }
  for (int k = 0; k < nfft; k++)
    if (prefac[k] < 1e-10) prefac[k] = 0.5 * (prefac[k - 1] + prefac[k + 1]);
  for (int k = 0; k < nfft; k++) prefac[k] = 1.0 / prefac[k];
  free(arr);
}

static void grid_anchor(double x, double recip, int nfft, int *i0, double *w) {
  double t = x * recip + 2.0;
  double fr = nfft * (t - (floor(t + 0.5) - 0.5));
  int fi = (int)fr;
  *i0 = fi;
  *w = fr - fi;
}

/*
 * Smooth PME reciprocal energy and gradient.  out virial6: xx, xy, xz, yy, yz,
 * zz of the reciprocal virial in the reference's sign convention.  The energy
 * sum adds the conjugate term for every k1 >= 1 of the half-complex grid, as
 * the reference does (so the k1 = nx/2 plane is counted twice).
 */
int or_pme(int n, const double *xyz, const double *q, const double *box,
           double kappa, int nx, int ny, int nz, int order, double *grad,
           double *energy, double *virial6, int nthreads) {
  set_threads(nthreads);
  size_t G = (size_t)nx * ny * nz;
  double *g = (double *)calloc(2 * G, sizeof(double));
  double *px = (double *)malloc(sizeof(double) * nx);
  double *py = (double *)malloc(sizeof(double) * ny);
  double *pz = (double *)malloc(sizeof(double) * nz);
  if (!g || !px || !py || !pz) return -1;
  bspline_moduli(nx, order, px);
  bspline_moduli(ny, order, py);
  bspline_moduli(nz, order, pz);
  double rx = 1.0 / box[0], ry = 1.0 / box[1], rz = 1.0 / box[2];
  /* spread (serial: deterministic) */
  for (int i = 0; i < n; i++) {
    int ix, iy, iz;
    double wx, wy, wz, tx[16], ty[16], tz[16], d[16];
    grid_anchor(xyz[3 * i], rx, nx, &ix, &wx);
    grid_anchor(xyz[3 * i + 1], ry, ny, &iy, &wy);
    grid_anchor(xyz[3 * i + 2], rz, nz, &iz, &wz);
    bspline(wx, order, tx, d);
    bspline(wy, order, ty, d);
    bspline(wz, order, tz, d);
    for (int c = 0; c < order; c++) {
      int z = (iz + c) % nz;
      for (int b = 0; b < order; b++) {
        int y = (iy + b) % ny;
        for (int a = 0; a < order; a++) {
          int x = (ix + a) % nx;
          g[2 * (x + (size_t)nx * (y + (size_t)ny * z))] += q[i] * tx[a] * ty[b] * tz[c];
        }
      }
    }
  }
  fft3d(g, nx, ny, nz, -1.0);
  double fac = PI * PI / (kappa * kappa);
  double piv_inv = rx * ry * rz / PI;
  int nf1 = nx / 2 + (nx % 2), nf2 = ny / 2 + (ny % 2), nf3 = nz / 2 + (nz % 2);
  double e = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
  /* influence function over the full grid; energy restricted to the
   * half-complex index set k1 <= nx/2 with conjugate doubling for k1 >= 1 */
#pragma omp parallel for reduction(+ : e, v0, v1, v2, v3, v4, v5)
  for (int k3 = 0; k3 < nz; k3++)
    for (int k2 = 0; k2 < ny; k2++)
      for (int k1 = 0; k1 < nx; k1++) {
        size_t pos = k1 + (size_t)nx * (k2 + (size_t)ny * k3);
        if (k1 == 0 && k2 == 0 && k3 == 0) {
          g[2 * pos] = g[2 * pos + 1] = 0.0;
          continue;
        }
        int m1 = k1 >= nf1 ? k1 - nx : k1;
        int m2 = k2 >= nf2 ? k2 - ny : k2;
        int m3 = k3 >= nf3 ? k3 - nz : k3;
        double mh1 = rx * m1, mh2 = ry * m2, mh3 = rz * m3;
        double msq = mh1 * mh1 + mh2 * mh2 + mh3 * mh3;
        double eterm = exp(-fac * msq) * piv_inv * px[k1] * py[k2] * pz[k3] / msq;
        if (k1 <= nx / 2) {
          double mult = k1 >= 1 ? 2.0 : 1.0;
          double t1 = mult * eterm * (g[2 * pos] * g[2 * pos] + g[2 * pos + 1] * g[2 * pos + 1]);
          double vt = 2.0 * (fac + 1.0 / msq);
          e += t1;
          v0 += t1 * (vt * mh1 * mh1 - 1.0);
          v1 += t1 * vt * mh1 * mh2;
          v2 += t1 * vt * mh1 * mh3;
          v3 += t1 * (vt * mh2 * mh2 - 1.0);
          v4 += t1 * vt * mh2 * mh3;
          v5 += t1 * (vt * mh3 * mh3 - 1.0);
        }
        g[2 * pos] *= eterm;
        g[2 * pos + 1] *= eterm;
      }
  *energy = 0.5 * CCELEC * e;
  if (virial6) {
    virial6[0] = -0.5 * CCELEC * v0;
    virial6[1] = -0.5 * CCELEC * v1;
    virial6[2] = -0.5 * CCELEC * v2;
    virial6[3] = -0.5 * CCELEC * v3;
    virial6[4] = -0.5 * CCELEC * v4;
    virial6[5] = -0.5 * CCELEC * v5;
  }
  fft3d(g, nx, ny, nz, +1.0);
  /* gather */
#pragma omp parallel for
  for (int i = 0; i < n; i++) {
    int ix, iy, iz;
    double wx, wy, wz, tx[16], ty[16], tz[16], dx[16], dy[16], dz[16];
    grid_anchor(xyz[3 * i], rx, nx, &ix, &wx);
    grid_anchor(xyz[3 * i + 1], ry, ny, &iy, &wy);
    grid_anchor(xyz[3 * i + 2], rz, nz, &iz, &wz);
    bspline(wx, order, tx, dx);
    bspline(wy, order, ty, dy);
    bspline(wz, order, tz, dz);
    double f1 = 0, f2 = 0, f3 = 0;
    for (int c = 0; c < order; c++) {
      int z = (iz + c) % nz;
      for (int b = 0; b < order; b++) {
        int y = (iy + b) % ny;
        for (int a = 0; a < order; a++) {
          int x = (ix + a) % nx;
          double phi = g[2 * (x + (size_t)nx * (y + (size_t)ny * z))];
          f1 += dx[a] * ty[b] * tz[c] * phi;
          f2 += tx[a] * dy[b] * tz[c] * phi;
          f3 += tx[a] * ty[b] * dz[c] * phi;
        }
      }
    }
    double qc = q[i] * CCELEC;
    grad[3 * i + 0] += qc * rx * nx * f1;
    grad[3 * i + 1] += qc * ry * ny * f2;
    grad[3 * i + 2] += qc * rz * nz * f3;
  }
  free(g);
  free(px);
  free(py);
  free(pz);
  return 0;
}

/*
 * Exact Ewald reciprocal sum (no mesh):
 *   E = ccelec/(2 pi V) sum_{m != 0, |k_d| <= kmax_d} exp(-pi^2 m^2/kappa^2)/m^2 |S(m)|^2
 * Used to state the mesh error of PME itself on small systems.
 */
int or_ewald_recip(int n, const double *xyz, const double *q, const double *box,
                   double kappa, int kx, int ky, int kz, double *grad,
                   double *energy, int nthreads) {
  set_threads(nthreads);
  double V = box[0] * box[1] * box[2];
  double fac = PI * PI / (kappa * kappa);
  double e = 0.0;
  int nk = (2 * kx + 1) * (2 * ky + 1) * (2 * kz + 1);
  double *gl = (double *)calloc((size_t)3 * n, sizeof(double));
#pragma omp parallel
  {
    double *gp = (double *)calloc((size_t)3 * n, sizeof(double));
    double *cs = (double *)malloc(sizeof(double) * 2 * n);
#pragma omp for reduction(+ : e) schedule(dynamic, 16)
    for (int t = 0; t < nk; t++) {
      int a = t % (2 * kx + 1) - kx;
      int b = (t / (2 * kx + 1)) % (2 * ky + 1) - ky;
      int c = t / ((2 * kx + 1) * (2 * ky + 1)) - kz;
      if (a == 0 && b == 0 && c == 0) continue;
      double m1 = a / box[0], m2 = b / box[1], m3 = c / box[2];
      double msq = m1 * m1 + m2 * m2 + m3 * m3;
      double pref = exp(-fac * msq) / msq / (2.0 * PI * V) * CCELEC;
      double sr = 0, si = 0;
      for (int i = 0; i < n; i++) {
        double ph = 2.0 * PI * (m1 * xyz[3 * i] + m2 * xyz[3 * i + 1] + m3 * xyz[3 * i + 2]);
        cs[2 * i] = cos(ph);
        cs[2 * i + 1] = sin(ph);
        sr += q[i] * cs[2 * i];
        si += q[i] * cs[2 * i + 1];
      }
      e += pref * (sr * sr + si * si);
      for (int i = 0; i < n; i++) {
        /* dE/dr_i = pref * 2 q_i * 2 pi m * (-sin*sr + cos*si) */
        double s = pref * 2.0 * q[i] * 2.0 * PI *
                   (-cs[2 * i + 1] * sr + cs[2 * i] * si);
        gp[3 * i] += s * m1;
        gp[3 * i + 1] += s * m2;
        gp[3 * i + 2] += s * m3;
      }
    }
#pragma omp critical
    for (int i = 0; i < 3 * n; i++) gl[i] += gp[i];
    free(gp);
    free(cs);
  }
  for (int i = 0; i < 3 * n; i++) grad[i] += gl[i];
  free(gl);
  *energy = e;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* bonded                                                                    */
/* ------------------------------------------------------------------------ */

/* E = kb (r - b0)^2 (bonds and Urey-Bradley), src/CudaBondedForce.cu:85-150 */
double or_bonds(int nb, const int *ij, const double *kb, const double *b0,
                const double *xyz, double *grad) {
  double e = 0;
  for (int p = 0; p < nb; p++) {
    int i = ij[2 * p], j = ij[2 * p + 1];
    double d[3];
    for (int k = 0; k < 3; k++) d[k] = xyz[3 * i + k] - xyz[3 * j + k];
    double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double db = r - b0[p];
    e += kb[p] * db * db;
    double f = 2.0 * kb[p] * db / r;
    for (int k = 0; k < 3; k++) {
      grad[3 * i + k] += f * d[k];
      grad[3 * j + k] -= f * d[k];
    }
  }
  return e;
}

/* E = ktheta (theta - theta0)^2, cos(theta) clamped to +-0.999 as in
 * src/CudaBondedForce.cu:223-300 */
double or_angles(int na, const int *ijk, const double *kt, const double *t0,
                 const double *xyz, double *grad) {
  double e = 0;
  for (int p = 0; p < na; p++) {
    int i = ijk[3 * p], j = ijk[3 * p + 1], k = ijk[3 * p + 2];
    double a[3], b[3];
    for (int d = 0; d < 3; d++) {
      a[d] = xyz[3 * i + d] - xyz[3 * j + d];
      b[d] = xyz[3 * k + d] - xyz[3 * j + d];
    }
    double ra = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double rb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    double ua[3], ub[3];
    for (int d = 0; d < 3; d++) {
      ua[d] = a[d] / ra;
      ub[d] = b[d] / rb;
    }
    double cst = ua[0] * ub[0] + ua[1] * ub[1] + ua[2] * ub[2];
    if (cst > 0.999) cst = 0.999;
    if (cst < -0.999) cst = -0.999;
    double th = acos(cst);
    double da = th - t0[p];
    e += kt[p] * da * da;
    double df = -2.0 * kt[p] * da / sqrt(1.0 - cst * cst);
    for (int d = 0; d < 3; d++) {
      double gi = df * (ub[d] - cst * ua[d]) / ra;
      double gk = df * (ua[d] - cst * ub[d]) / rb;
      grad[3 * i + d] += gi;
      grad[3 * k + d] += gk;
      grad[3 * j + d] -= gi + gk;
    }
  }
  return e;
}

/*
 * Proper (harmonic == 0) and improper (harmonic == 1) dihedrals,
 * src/CudaBondedForce.cu:387-700.  Term t of dihedral p is
 * (k, n, delta) at term_ptr[p] .. term_ptr[p+1]-1; harmonic terms use
 * E = k (phi - delta)^2 (the reference's n == 0 improper branch).
 */
double or_dihedrals(int nd, const int *ijkl, const int *term_ptr,
                    const double *tk, const int *tn, const double *tdelta,
                    int harmonic, const double *xyz, double *grad) {
  double e = 0;
  for (int p = 0; p < nd; p++) {
    int i = ijkl[4 * p], j = ijkl[4 * p + 1], k = ijkl[4 * p + 2], l = ijkl[4 * p + 3];
    double F[3], Gv[3], H[3], A[3], B[3];
    for (int d = 0; d < 3; d++) {
      F[d] = xyz[3 * i + d] - xyz[3 * j + d];
      Gv[d] = xyz[3 * j + d] - xyz[3 * k + d];
      H[d] = xyz[3 * l + d] - xyz[3 * k + d];
    }
    A[0] = F[1] * Gv[2] - F[2] * Gv[1];
    A[1] = F[2] * Gv[0] - F[0] * Gv[2];
    A[2] = F[0] * Gv[1] - F[1] * Gv[0];
    B[0] = H[1] * Gv[2] - H[2] * Gv[1];
    B[1] = H[2] * Gv[0] - H[0] * Gv[2];
    B[2] = H[0] * Gv[1] - H[1] * Gv[0];
    double ra2 = A[0] * A[0] + A[1] * A[1] + A[2] * A[2];
    double rb2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    double rg = sqrt(Gv[0] * Gv[0] + Gv[1] * Gv[1] + Gv[2] * Gv[2]);
    double rabr = 1.0 / sqrt(ra2 * rb2);
    double ct = (A[0] * B[0] + A[1] * B[1] + A[2] * B[2]) * rabr;
    double st = rg * rabr * (A[0] * H[0] + A[1] * H[1] + A[2] * H[2]);
    double phi = atan2(st, ct);
    double df = 0.0;
    for (int t = term_ptr[p]; t < term_ptr[p + 1]; t++) {
      if (harmonic) {
        double ap = phi - tdelta[t];
        while (ap > PI) ap -= 2 * PI;
        while (ap < -PI) ap += 2 * PI;
        e += tk[t] * ap * ap;
        df += 2.0 * tk[t] * ap;
      } else {
        int nn = tn[t];
        e += tk[t] * (1.0 + cos(nn * phi - tdelta[t]));
        df += -tk[t] * nn * sin(nn * phi - tdelta[t]);
      }
    }
    double fg = F[0] * Gv[0] + F[1] * Gv[1] + F[2] * Gv[2];
    double hg = H[0] * Gv[0] + H[1] * Gv[1] + H[2] * Gv[2];
    double ra2r = df / ra2, rb2r = df / rb2;
    double fga = fg * ra2r / rg, hgb = hg * rb2r / rg;
    double gaa = ra2r * rg, gbb = rb2r * rg;
    for (int d = 0; d < 3; d++) {
      double dfv = -gaa * A[d];
      double dgv = fga * A[d] - hgb * B[d];
      double dhv = gbb * B[d];
      grad[3 * i + d] += dfv;
      grad[3 * j + d] += dgv - dfv;
      grad[3 * k + d] += -dhv - dgv;
      grad[3 * l + d] += dhv;
    }
  }
  return e;
}
