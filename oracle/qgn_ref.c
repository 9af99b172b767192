/*
 * qgn_ref.c -- C / OpenMP FP64 restatement of QGN's spectral RHS and time steppers.
 *
 * TEST INFRASTRUCTURE ONLY: the CPU oracle at large sizes and the timed CPU baseline
 * (bench.py's cpu_baseline and --impl reference legs).  It is never called by the product.
 *
 * Parity status: UNPINNED (the reference is Fortran + Intel MKL, neither available where this
 * project builds; the reference ships no tests or golden data).  It is cross-checked against
 * the numpy restatement oracle/qgn_oracle.py in tests/test_oracle_c.py.
 *
 * It follows the reference routine by routine on full arrays (no compact storage):
 *   DeAlias        QGN_Module.f90:194-204      GetPsi   QGN_Module.f90:315-341
 *   Jacobian       QGN_Module.f90:215-249      GetRHS   QGN_Module.f90:258-296
 *   ARK43_QGLeith.f90, ARK43.f90, BSRK3.f90, RK4.f90, AB3.f90
 * with its own FFT in place of MKL DFTI (MKL_DFTI_Setup.f90): iterative radix-2 complex
 * transforms; rows of the real 2-D transforms are paired into one complex transform
 * (f1 + i f2); c2r applies the y transform first and keeps Re of the kx=0 (and Nyquist)
 * entry, the Hermitian projection of a y-then-x c2r.  Layout: spectral [nz][ny][nx/2+1]
 * complex (= Fortran q_hat(nx/2+1,ny,nz)), physical [nz][ny][nx] (= q(nx,ny,nz)).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

typedef struct {
    int nx, ny, nz, nxh, scheme, is_explicit;
    double Lx, Ly, Htot, beta, A2, A8, r0, C_d, TOL, dt_max;
    double *H, *uBar, *qyBar, *Modes, *EVals; /* Modes column-major nz x nz */
    double *kx, *ky, *k2;                     /* [ny][nxh] */
    cplx *twx, *twy;                          /* exp(-2 pi i m / n), m < n/2 */
    int *revx, *revy;
    /* work arrays (full spectral / physical) */
    cplx *psi, *uh, *vh, *spec, *jac;
    double *qp, *up, *vp, *gp;
    /* stepper memory */
    cplx *N[6], *L[6], *qtmp, *Mq, *save0, *save1;
    double err0;
    int first, calls;
    long long rejects;
} qgn_ref;

/* ---------------------------------------------------------------------------- FFT */
static int ilog2i(int n) { int k = 0; while ((1 << k) < n) ++k; return k; }

static void make_fft(int n, cplx** tw, int** rev) {
    *tw = (cplx*)malloc(sizeof(cplx) * (n / 2 > 0 ? n / 2 : 1));
    *rev = (int*)malloc(sizeof(int) * n);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < n / 2; ++m) {
        long double a = 2.0L * PI * (long double)m / (long double)n;
        (*tw)[m] = (double)cosl(a) - I * (double)sinl(a);
    }
    int lg = ilog2i(n);
    for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
        (*rev)[i] = r;
    }
}

/* in-place radix-2 DIT FFT of length n; sign -1 forward, +1 backward (unnormalised) */
static void fft1(cplx* a, int n, const cplx* tw, const int* rev, int sign) {
    for (int i = 0; i < n; ++i) {
        int j = rev[i];
        if (j > i) { cplx t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; ++k) {
                cplx w = tw[k * step];
                if (sign > 0) w = conj(w);
                cplx u = a[s + k], v = a[s + k + half] * w;
                a[s + k] = u + v;
                a[s + k + half] = u - v;
            }
        }
    }
}

/* batched 2-D r2c: g[nz][ny][nx] -> s[nz][ny][nxh] (unnormalised, DftiComputeForward) */
static void r2c2(const qgn_ref* m, const double* g, cplx* s) {
    const int nx = m->nx, ny = m->ny, nz = m->nz, nxh = m->nxh;
#pragma omp parallel
    {
        cplx* row = (cplx*)malloc(sizeof(cplx) * (nx > ny ? nx : ny));
#pragma omp for collapse(2) schedule(static)
        for (int l = 0; l < nz; ++l)
            for (int p = 0; p < ny / 2; ++p) {
                const double* r1 = g + ((size_t)l * ny + 2 * p) * nx;
                const double* r2 = r1 + nx;
                for (int x = 0; x < nx; ++x) row[x] = r1[x] + I * r2[x];
                fft1(row, nx, m->twx, m->revx, -1);
                cplx* o1 = s + ((size_t)l * ny + 2 * p) * nxh;
                cplx* o2 = o1 + nxh;
                for (int k = 0; k < nxh; ++k) {
                    cplx X = row[k], Y = conj(row[(nx - k) % nx]);
                    o1[k] = 0.5 * (X + Y);
                    o2[k] = -0.5 * I * (X - Y);
                }
            }
#pragma omp for collapse(2) schedule(static)
        for (int l = 0; l < nz; ++l)
            for (int k = 0; k < nxh; ++k) {
                cplx* c = s + (size_t)l * ny * nxh + k;
                for (int j = 0; j < ny; ++j) row[j] = c[(size_t)j * nxh];
                fft1(row, ny, m->twy, m->revy, -1);
                for (int j = 0; j < ny; ++j) c[(size_t)j * nxh] = row[j];
            }
        free(row);
    }
}

/* batched 2-D c2r scaled by 1/(nx ny): s[nz][ny][nxh] -> g (DftiComputeBackward + grid/(nx*ny)) */
static void c2r2(const qgn_ref* m, const cplx* s_in, double* g, cplx* work) {
    const int nx = m->nx, ny = m->ny, nz = m->nz, nxh = m->nxh;
    const double sc = 1.0 / ((double)nx * (double)ny);
    memcpy(work, s_in, sizeof(cplx) * (size_t)nz * ny * nxh);
#pragma omp parallel
    {
        cplx* row = (cplx*)malloc(sizeof(cplx) * (nx > ny ? nx : ny));
#pragma omp for collapse(2) schedule(static)
        for (int l = 0; l < nz; ++l)
            for (int k = 0; k < nxh; ++k) {
                cplx* c = work + (size_t)l * ny * nxh + k;
                for (int j = 0; j < ny; ++j) row[j] = c[(size_t)j * nxh];
                fft1(row, ny, m->twy, m->revy, +1);
                for (int j = 0; j < ny; ++j) c[(size_t)j * nxh] = row[j];
            }
#pragma omp for collapse(2) schedule(static)
        for (int l = 0; l < nz; ++l)
            for (int p = 0; p < ny / 2; ++p) {
                const cplx* F1 = work + ((size_t)l * ny + 2 * p) * nxh;
                const cplx* F2 = F1 + nxh;
                for (int k = 0; k < nx; ++k) row[k] = 0.0;
                for (int k = 0; k < nxh; ++k) {
                    cplx a = F1[k], b = F2[k];
                    if (k == 0 || 2 * k == nx) { a = creal(a); b = creal(b); }
                    row[k] = a + I * b;
                    if (k > 0 && 2 * k < nx) row[nx - k] = conj(a) + I * conj(b);
                }
                fft1(row, nx, m->twx, m->revx, +1);
                double* o1 = g + ((size_t)l * ny + 2 * p) * nx;
                double* o2 = o1 + nx;
                for (int x = 0; x < nx; ++x) { o1[x] = creal(row[x]) * sc; o2[x] = cimag(row[x]) * sc; }
            }
        free(row);
    }
}

/* ------------------------------------------------------------------------ the model */
static size_t SZ(const qgn_ref* m) { return (size_t)m->nz * m->ny * m->nxh; }
static size_t PZ(const qgn_ref* m) { return (size_t)m->nz * m->ny * m->nx; }

static void dealias(const qgn_ref* m, cplx* f) {
    const int nx = m->nx, ny = m->ny, nxh = m->nxh;
#pragma omp parallel for collapse(2)
    for (int l = 0; l < m->nz; ++l)
        for (int j = 0; j < ny; ++j) {
            cplx* r = f + ((size_t)l * ny + j) * nxh;
            if (j >= ny / 3 && j <= 2 * (ny / 3)) {
                for (int i = 0; i < nxh; ++i) r[i] = 0.0;
            } else {
                for (int i = nx / 3; i < nxh; ++i) r[i] = 0.0;
            }
            if (j == 0) r[0] = 0.0;
        }
}

static void get_psi(qgn_ref* m, const cplx* q) {
    const int nz = m->nz;
    const size_t P = (size_t)m->ny * m->nxh;
#pragma omp parallel for schedule(static)
    for (size_t p = 0; p < P; ++p) {
        cplx qm[64], pm[64];
        for (int k = 0; k < nz; ++k) {
            cplx acc = 0.0;
            for (int kk = 0; kk < nz; ++kk) acc += (m->H[kk] * m->Modes[kk + (size_t)k * nz]) * q[(size_t)kk * P + p];
            qm[k] = acc / m->Htot;
            pm[k] = (p == 0) ? 0.0 : qm[k] / (-m->k2[p] + m->EVals[k]);
        }
        for (int k = 0; k < nz; ++k) {
            cplx acc = 0.0;
            for (int kk = 0; kk < nz; ++kk) acc += pm[kk] * m->Modes[k + (size_t)kk * nz];
            m->psi[(size_t)k * P + p] = acc;
        }
    }
}

static void get_rhs(qgn_ref* m, const cplx* q, cplx* rhs) {
    const int nz = m->nz;
    const size_t P = (size_t)m->ny * m->nxh;
    const size_t S = SZ(m), NP = PZ(m);
    get_psi(m, q);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < S; ++e) {
        size_t p = e % P;
        m->uh[e] = -I * m->ky[p] * m->psi[e];
        m->vh[e] = I * m->kx[p] * m->psi[e];
    }
    c2r2(m, q, m->qp, m->spec);
    c2r2(m, m->uh, m->up, m->spec);
    c2r2(m, m->vh, m->vp, m->spec);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < NP; ++e) m->gp[e] = m->up[e] * m->qp[e];
    r2c2(m, m->gp, m->jac);                          /* uq_hat */
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < NP; ++e) m->gp[e] = m->vp[e] * m->qp[e];
    r2c2(m, m->gp, m->spec);                         /* vq_hat */
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < S; ++e) {
        size_t p = e % P;
        int k = (int)(e / P);
        cplx jac = I * m->kx[p] * m->jac[e] + I * m->ky[p] * m->spec[e];
        cplx r = -jac;
        r = r - m->uBar[k] * I * m->kx[p] * q[e] - (m->beta + m->qyBar[k]) * m->vh[e];
        if (m->is_explicit) {
            double k2 = m->k2[p], k8 = (k2 * k2) * (k2 * k2);
            r = r - (m->A2 * k2 + m->A8 * k8) * q[e];
        }
        rhs[e] = r;
    }
    const size_t bot = (size_t)(nz - 1) * P;
    const double ek = m->r0 * m->Htot / m->H[nz - 1];
    for (size_t p = 0; p < P; ++p) rhs[bot + p] += ek * m->k2[p] * m->psi[bot + p];
    if (m->C_d != 0.0) {
        /* |u|u and |u|v over all layers (only the bottom layer is used, QGN_Module.f90:284-292) */
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < NP; ++e) {
            double urms = sqrt(m->up[e] * m->up[e] + m->vp[e] * m->vp[e]);
            m->gp[e] = urms * m->up[e];
        }
        r2c2(m, m->gp, m->jac);
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < NP; ++e) {
            double urms = sqrt(m->up[e] * m->up[e] + m->vp[e] * m->vp[e]);
            m->gp[e] = urms * m->vp[e];
        }
        r2c2(m, m->gp, m->spec);
        const double dc = m->C_d * m->Htot / m->H[nz - 1];
        for (size_t p = 0; p < P; ++p) {
            cplx d = I * m->ky[p] * m->jac[bot + p] - I * m->kx[p] * m->spec[bot + p];
            rhs[bot + p] += dc * d;
        }
    }
    dealias(m, rhs);
}

/* ------------------------------------------------------------------------- steppers */
static const double AE[6][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.5, 0, 0, 0, 0, 0},
    {13861.0 / 62500.0, 6889.0 / 62500.0, 0, 0, 0, 0},
    {-116923316275.0 / 2393684061468.0, -2731218467317.0 / 15368042101831.0, 9408046702089.0 / 11113171139209.0, 0, 0, 0},
    {-451086348788.0 / 2902428689909.0, -2682348792572.0 / 7519795681897.0, 12662868775082.0 / 11960479115383.0,
     3355817975965.0 / 11060851509271.0, 0, 0},
    {647845179188.0 / 3216320057751.0, 73281519250.0 / 8382639484533.0, 552539513391.0 / 3454668386233.0,
     3354512671639.0 / 8306763924573.0, 4040.0 / 17871.0, 0}};
static const double BB[6] = {82889.0 / 524892.0, 0.0, 15625.0 / 83664.0, 69875.0 / 102672.0, -2260.0 / 8211.0, 0.25};
static const double AI[6][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.25, 0.25, 0, 0, 0, 0},
    {8611.0 / 62500.0, -1743.0 / 31250.0, 0, 0, 0, 0},
    {5012029.0 / 34652500.0, -654441.0 / 2922500.0, 174375.0 / 388108.0, 0, 0, 0},
    {15267082809.0 / 155376265600.0, -71443401.0 / 120774400.0, 730878875.0 / 902184768.0, 2285395.0 / 8070912.0, 0, 0},
    {82889.0 / 524892.0, 0.0, 15625.0 / 83664.0, 69875.0 / 102672.0, -2260.0 / 8211.0, 0.25}};
static const double BE[6] = {31666707.0 / 9881966720.0, 0.0, -256875.0 / 105007616.0, -2768025.0 / 128864768.0,
                             169839.0 / 3864644.0, -5247.0 / 225920.0};

static double maxabs_phys(qgn_ref* m, const cplx* spec) {
    c2r2(m, spec, m->gp, m->spec);
    const size_t NP = PZ(m);
    double mx = 0.0;
#pragma omp parallel for reduction(max : mx)
    for (size_t e = 0; e < NP; ++e) {
        double a = fabs(m->gp[e]);
        if (a > mx) mx = a;
    }
    return mx * ((double)m->nx * (double)m->ny);   /* undo the 1/(nx ny): MAXVAL(ABS(grid)) */
}

/* returns 0 ok, 4 reject limit */
static int step_ark(qgn_ref* m, cplx* q, double* t, double* dt, int leith, int max_rejects) {
    const int nz = m->nz;
    const size_t P = (size_t)m->ny * m->nxh, S = SZ(m);
    double A8L[64];
    if (leith) {
        /* ARK43_QGLeith.f90:62-73 in physical space */
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < S; ++e) {
            double k2 = m->k2[e % P];
            m->uh[e] = ((k2 * k2) * (k2 * k2)) * q[e];
        }
        c2r2(m, m->uh, m->up, m->spec);
        c2r2(m, q, m->qp, m->spec);
        const double x = (double)1.3f * m->Lx / ((double)m->nx * (4.0 * atan(1.0)));
        const double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, c12 = x4 * x8;
        const size_t NP1 = (size_t)m->ny * m->nx;
        for (int k = 0; k < nz; ++k) {
            double s = 0.0;
#pragma omp parallel for reduction(+ : s)
            for (size_t e = 0; e < NP1; ++e) s += m->qp[(size_t)k * NP1 + e] * m->up[(size_t)k * NP1 + e];
            A8L[k] = c12 * sqrt(s / ((double)m->nx * m->ny));
        }
    } else {
        for (int k = 0; k < nz; ++k) A8L[k] = m->A8;
    }
    get_rhs(m, q, m->N[0]);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < S; ++e) {
        double k2 = m->k2[e % P], k8 = (k2 * k2) * (k2 * k2);
        m->L[0][e] = -(m->A2 * k2 + A8L[e / P] * k8) * q[e];
    }
    const double rfac = leith ? 0.5 : 0.75, safety = leith ? 0.2 : 0.75;
    for (int nrej = 0;;) {
        const double dtv = *dt;
        for (int s = 1; s < 6; ++s) {
#pragma omp parallel for schedule(static)
            for (size_t e = 0; e < S; ++e) {
                double k2 = m->k2[e % P], k8 = (k2 * k2) * (k2 * k2);
                double D = m->A2 * k2 + A8L[e / P] * k8;
                cplx acc = AE[s][0] * m->N[0][e];
                for (int j = 1; j < s; ++j) acc += AE[s][j] * m->N[j][e];
                for (int j = 0; j < s; ++j) acc += AI[s][j] * m->L[j][e];
                m->qtmp[e] = (1.0 / (1.0 + 0.25 * dtv * D)) * (q[e] + dtv * acc);
            }
            get_rhs(m, m->qtmp, m->N[s]);
#pragma omp parallel for schedule(static)
            for (size_t e = 0; e < S; ++e) {
                double k2 = m->k2[e % P], k8 = (k2 * k2) * (k2 * k2);
                m->L[s][e] = -(m->A2 * k2 + A8L[e / P] * k8) * m->qtmp[e];
            }
        }
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < S; ++e) {
            cplx v = BE[0] * (m->N[0][e] + m->L[0][e]);
            for (int i = 2; i < 6; ++i) v += BE[i] * (m->N[i][e] + m->L[i][e]);
            m->save0[e] = v;
        }
        const double err1 = dtv * maxabs_phys(m, m->save0) / ((double)m->nx * m->ny);
        if (err1 > m->TOL) {
            *dt = rfac * dtv;
            ++m->rejects;
            if (++nrej >= max_rejects) return 4;
            continue;
        }
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < S; ++e) {
            cplx v = BB[0] * (m->N[0][e] + m->L[0][e]);
            for (int i = 2; i < 6; ++i) v += BB[i] * (m->N[i][e] + m->L[i][e]);
            q[e] = (e % P == 0) ? 0.0 : q[e] + dtv * v;
        }
        *t += dtv;
        double nd = dtv * pow(safety * m->TOL / err1, 0.075) * pow(m->err0 / err1, 0.1);
        *dt = nd < m->dt_max ? nd : m->dt_max;
        m->err0 = err1;
        return 0;
    }
}

static void axpy(const qgn_ref* m, cplx* out, const cplx* q, int n, const double* c, cplx* const* R) {
    const size_t S = SZ(m);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < S; ++e) {
        cplx v = q[e];
        for (int j = 0; j < n; ++j) v += c[j] * R[j][e];
        out[e] = v;
    }
}

static int step_bsrk3(qgn_ref* m, cplx* q, double* t, double* dt, int max_rejects) {
    if (m->first) {
        get_rhs(m, q, m->N[0]);
        m->err0 = m->TOL;
        m->first = 0;
    }
    for (int nrej = 0;;) {
        const double d = *dt;
        double c1[1] = {0.5 * d};
        axpy(m, m->qtmp, q, 1, c1, &m->N[0]);
        get_rhs(m, m->qtmp, m->N[1]);
        double c2[1] = {0.75 * d};
        axpy(m, m->qtmp, q, 1, c2, &m->N[1]);
        get_rhs(m, m->qtmp, m->N[2]);
        double c3[3] = {2.0 * d / 9.0, 1.0 * d / 3.0, 4.0 * d / 9.0};
        axpy(m, m->qtmp, q, 3, c3, m->N);
        get_rhs(m, m->qtmp, m->N[3]);
        const size_t S = SZ(m);
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < S; ++e)
            m->save0[e] = (5.0 / 72.0) * m->N[0][e] - (1.0 / 12.0) * m->N[1][e] - (1.0 / 9.0) * m->N[2][e] +
                          (1.0 / 8.0) * m->N[3][e];
        const double r1 = d * (maxabs_phys(m, m->save0) / ((double)m->nx * m->ny));
        if (r1 > m->TOL) {
            *dt = 0.75 * d;
            ++m->rejects;
            if (++nrej >= max_rejects) return 4;
            continue;
        }
        memcpy(q, m->qtmp, sizeof(cplx) * S);
        *t += d;
        cplx* tmp = m->N[0];
        m->N[0] = m->N[3];
        m->N[3] = tmp;
        double nd = d * pow(0.75 * m->TOL / r1, 0.1) * pow(m->err0 / r1, 0.4 / 3.0);
        *dt = nd < m->dt_max ? nd : m->dt_max;
        m->err0 = r1;
        return 0;
    }
}

static int step_rk4(qgn_ref* m, cplx* q, double* t, double* dt) {
    const double d = *dt;
    get_rhs(m, q, m->N[0]);
    double c[1] = {0.5 * d};
    axpy(m, m->qtmp, q, 1, c, &m->N[0]);
    get_rhs(m, m->qtmp, m->N[1]);
    axpy(m, m->qtmp, q, 1, c, &m->N[1]);
    get_rhs(m, m->qtmp, m->N[2]);
    double c3[1] = {d};
    axpy(m, m->qtmp, q, 1, c3, &m->N[2]);
    get_rhs(m, m->qtmp, m->N[3]);
    const size_t S = SZ(m);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < S; ++e)
        q[e] = q[e] + (d / 6.0) * (m->N[0][e] + 2.0 * m->N[1][e] + 2.0 * m->N[2][e] + m->N[3][e]);
    *t += d;
    return 0;
}

static int step_ab3(qgn_ref* m, cplx* q, double* t, double* dt) {
    const double d = *dt;
    const size_t S = SZ(m);
    if (m->calls == 0) {
        get_rhs(m, q, m->save0);
#pragma omp parallel for
        for (size_t e = 0; e < S; ++e) q[e] = q[e] + d * m->save0[e];
    } else if (m->calls == 1) {
        get_rhs(m, q, m->save1);
#pragma omp parallel for
        for (size_t e = 0; e < S; ++e) q[e] = q[e] + d * (1.5 * m->save1[e] - 0.5 * m->save0[e]);
    } else {
        get_rhs(m, q, m->N[0]);
#pragma omp parallel for
        for (size_t e = 0; e < S; ++e)
            q[e] = q[e] + (d / 12.0) * (23.0 * m->N[0][e] - 16.0 * m->save1[e] + 5.0 * m->save0[e]);
        cplx* t0 = m->save0;
        m->save0 = m->save1;
        m->save1 = m->N[0];
        m->N[0] = t0;
    }
    ++m->calls;
    *t += d;
    return 0;
}

/* ---------------------------------------------------------------------------- C-ABI */
void* qgn_ref_create(int nx, int ny, int nz, int scheme, int is_explicit, const double* prm /* Lx Ly Htot beta A2 A8 r0 C_d TOL dt_max */,
                     const double* H, const double* uBar, const double* qyBar, const double* Modes, const double* EVals) {
    qgn_ref* m = (qgn_ref*)calloc(1, sizeof(qgn_ref));
    m->nx = nx; m->ny = ny; m->nz = nz; m->nxh = nx / 2 + 1; m->scheme = scheme; m->is_explicit = is_explicit;
    m->Lx = prm[0]; m->Ly = prm[1]; m->Htot = prm[2]; m->beta = prm[3]; m->A2 = prm[4]; m->A8 = prm[5];
    m->r0 = prm[6]; m->C_d = prm[7]; m->TOL = prm[8]; m->dt_max = prm[9];
    m->H = (double*)malloc(sizeof(double) * nz); memcpy(m->H, H, sizeof(double) * nz);
    m->uBar = (double*)malloc(sizeof(double) * nz); memcpy(m->uBar, uBar, sizeof(double) * nz);
    m->qyBar = (double*)malloc(sizeof(double) * nz); memcpy(m->qyBar, qyBar, sizeof(double) * nz);
    m->Modes = (double*)malloc(sizeof(double) * nz * nz); memcpy(m->Modes, Modes, sizeof(double) * nz * nz);
    m->EVals = (double*)malloc(sizeof(double) * nz); memcpy(m->EVals, EVals, sizeof(double) * nz);
    const size_t P = (size_t)ny * m->nxh, S = SZ(m), NP = PZ(m);
    m->kx = (double*)malloc(sizeof(double) * P); m->ky = (double*)malloc(sizeof(double) * P);
    m->k2 = (double*)malloc(sizeof(double) * P);
    const double pi = 4.0 * atan(1.0);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < m->nxh; ++i) {
            size_t p = (size_t)j * m->nxh + i;
            m->kx[p] = (2.0 * pi / m->Lx) * (double)i;
            m->ky[p] = (2.0 * pi / m->Ly) * (double)(j <= ny / 2 ? j : j - ny);
            m->k2[p] = m->kx[p] * m->kx[p] + m->ky[p] * m->ky[p];
        }
    make_fft(nx, &m->twx, &m->revx);
    make_fft(ny, &m->twy, &m->revy);
    m->psi = (cplx*)malloc(sizeof(cplx) * S); m->uh = (cplx*)malloc(sizeof(cplx) * S);
    m->vh = (cplx*)malloc(sizeof(cplx) * S); m->spec = (cplx*)malloc(sizeof(cplx) * S);
    m->jac = (cplx*)malloc(sizeof(cplx) * S);
    m->qp = (double*)malloc(sizeof(double) * NP); m->up = (double*)malloc(sizeof(double) * NP);
    m->vp = (double*)malloc(sizeof(double) * NP); m->gp = (double*)malloc(sizeof(double) * NP);
    for (int i = 0; i < 6; ++i) { m->N[i] = (cplx*)malloc(sizeof(cplx) * S); m->L[i] = (cplx*)malloc(sizeof(cplx) * S); }
    m->qtmp = (cplx*)malloc(sizeof(cplx) * S); m->Mq = (cplx*)malloc(sizeof(cplx) * S);
    m->save0 = (cplx*)malloc(sizeof(cplx) * S); m->save1 = (cplx*)malloc(sizeof(cplx) * S);
    m->err0 = m->TOL;
    m->first = 1;
    return m;
}

void qgn_ref_destroy(void* h) {
    qgn_ref* m = (qgn_ref*)h;
    if (!m) return;
    void* ps[] = {m->H, m->uBar, m->qyBar, m->Modes, m->EVals, m->kx, m->ky, m->k2, m->twx, m->twy, m->revx, m->revy,
                  m->psi, m->uh, m->vh, m->spec, m->jac, m->qp, m->up, m->vp, m->gp, m->qtmp, m->Mq, m->save0, m->save1};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
    for (int i = 0; i < 6; ++i) { free(m->N[i]); free(m->L[i]); }
    free(m);
}

void qgn_ref_rhs(void* h, const double* q, double* rhs) { get_rhs((qgn_ref*)h, (const cplx*)q, (cplx*)rhs); }

void qgn_ref_forward(void* h, const double* phys, double* spec) {
    qgn_ref* m = (qgn_ref*)h;
    r2c2(m, phys, (cplx*)spec);
    dealias(m, (cplx*)spec);
}

/* one TimeStep (the scheme include + DeAlias, QGN_Module.f90:302-309); returns 0 or 4 */
int qgn_ref_step(void* h, double* q, double* t, double* dt, int max_rejects) {
    qgn_ref* m = (qgn_ref*)h;
    cplx* qc = (cplx*)q;
    int rc;
    switch (m->scheme) {
        case 0: rc = step_ark(m, qc, t, dt, 1, max_rejects); break;
        case 1: rc = step_ark(m, qc, t, dt, 0, max_rejects); break;
        case 2: rc = step_bsrk3(m, qc, t, dt, max_rejects); break;
        case 3: rc = step_rk4(m, qc, t, dt); break;
        default: rc = step_ab3(m, qc, t, dt); break;
    }
    dealias(m, qc);
    return rc;
}

long long qgn_ref_rejects(void* h) { return ((qgn_ref*)h)->rejects; }

int qgn_ref_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
