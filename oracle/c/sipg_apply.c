/*
 * Oracle (test infrastructure, CPU baseline only): float64 SIPG apply,
 * C + OpenMP.  Restates the derivative of ddg's sipg_bilinear_form
 * (src/ddg/dg2d/sipg.py:142-337, affine branch) with the reference's own
 * per-node arrays: geometric factors (Np, K), face normals / sJ / Fscale
 * (3 Nfp, K) and the vmapM / vmapP node maps (src/ddg/dg2d/mesh.py:574-627).
 *
 * Every element computes all contributions to its own nodes: the ones the
 * reference adds from its own face traces and the ones it scatters from the
 * neighbouring element through vmapP (interior faces carry w = 1/2 from each
 * side, sipg.py:135-138), so the element loop is parallel without atomics.
 * Not used by the GPU product.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NFMAX 8
#define NPMAX 45

typedef struct {
    int N, Np, Nfp, K;
    const double *Dr, *Ds, *M, *m1d;        /* (Np,Np) row-major, m1d (3,Nfp,Nfp) */
    const int64_t *Fmask;                    /* (Nfp,3) */
    const double *rx, *sx, *ry, *sy, *J;     /* (Np,K) row-major */
    const double *nx, *ny, *sJ, *Fscale;     /* (3Nfp,K) row-major */
    const int64_t *vmapM, *vmapP;            /* (3 Nfp K) */
    const int64_t *EToE, *EToF;              /* (K,3) */
    const int32_t *bc;                       /* (K,3) */
    double tau_scale, alpha;
} oracle_mesh;

/* physical gradient of element k's field at local node n */
static void grad_at(const oracle_mesh *m, const double *u, int64_t k, int n, double *gx, double *gy) {
    const int Np = m->Np;
    const double *uk = u + k * Np;
    double ar = 0.0, as = 0.0;
    for (int j = 0; j < Np; ++j) {
        ar += m->Dr[n * Np + j] * uk[j];
        as += m->Ds[n * Np + j] * uk[j];
    }
    const int64_t K = m->K;
    *gx = m->rx[n * K + k] * ar + m->sx[n * K + k] * as;
    *gy = m->ry[n * K + k] * ar + m->sy[n * K + k] * as;
}

void oracle_sipg_apply(const oracle_mesh *m, const double *u, double *y, int nthreads) {
    const int Np = m->Np, Nfp = m->Nfp, N = m->N;
    const int64_t K = m->K;
    const double tau0 = m->tau_scale * (N + 1) * (N + 1);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t k = 0; k < K; ++k) {
        double ux[NPMAX], uy[NPMAX], ex[NPMAX], ey[NPMAX], yk[NPMAX];
        const double *uk = u + k * Np;
        for (int n = 0; n < Np; ++n) grad_at(m, u, k, n, &ux[n], &uy[n]);
        for (int i = 0; i < Np; ++i) {
            double a = 0.0, b = 0.0, c = 0.0;
            for (int j = 0; j < Np; ++j) {
                a += m->M[j * Np + i] * m->J[j * K + k] * ux[j];
                b += m->M[j * Np + i] * m->J[j * K + k] * uy[j];
                c += m->M[i * Np + j] * uk[j];
            }
            ex[i] = a;
            ey[i] = b;
            yk[i] = m->alpha * m->J[i * K + k] * c;
        }
        for (int f = 0; f < 3; ++f) {
            const int tag = m->bc[k * 3 + f];
            const int64_t kp = m->EToE[k * 3 + f], fp = m->EToF[k * 3 + f];
            const int self = (kp == k && fp == f);
            const int tagp = self ? -1 : m->bc[kp * 3 + fp];
            /* weights: own side (M) and neighbour side (P, scattered through vmapP) */
            const int mdir = (tag == 1), mint = (tag == 0 && !self), pact = (!self && tagp == 0);
            if (!(mdir || mint || pact)) continue;
            const int64_t base = (k * 3 + f) * Nfp;
            const double sJf = m->sJ[(f * Nfp) * K + k];
            const double tauM = tau0 * m->Fscale[(f * Nfp) * K + k];
            double tauP = tauM;
            if (!self) tauP = tau0 * m->Fscale[(fp * Nfp) * K + kp];
            double v1[NFMAX], v2[NFMAX];
            for (int p = 0; p < Nfp; ++p) {
                const int64_t iM = m->vmapM[base + p], iP = m->vmapP[base + p];
                const int nM = (int)(iM % Np), nP = (int)(iP % Np);
                const int64_t kP = iP / Np;
                const double nxv = m->nx[(f * Nfp + p) * K + k], nyv = m->ny[(f * Nfp + p) * K + k];
                const double uM = u[iM], uP = u[iP];
                double gxP, gyP;
                grad_at(m, u, kP, nP, &gxP, &gyP);
                const double dnM = nxv * ux[nM] + nyv * uy[nM];
                const double dnP = nxv * gxP + nyv * gyP;
                const double avgI = 0.5 * (dnM + dnP), jmpI = uM - uP;
                const double avgM = mdir ? dnM : avgI, jmpM = mdir ? uM : jmpI;
                const double caM = mdir ? 1.0 : (mint ? 0.5 : 0.0);
                const double cjM = mdir ? tauM : (mint ? 0.5 * tauM : 0.0);
                const double cgM = mdir ? 1.0 : (mint ? 0.25 : 0.0);
                const double caP = pact ? 0.5 : 0.0, cjP = pact ? 0.5 * tauP : 0.0, cgP = pact ? 0.25 : 0.0;
                v1[p] = -caM * avgM + cjM * jmpM - caP * avgI + cjP * jmpI;
                v2[p] = cgM * jmpM + cgP * jmpI;
            }
            for (int q = 0; q < Nfp; ++q) {
                double a = 0.0, b = 0.0;
                for (int p = 0; p < Nfp; ++p) {
                    a += m->m1d[(f * Nfp + p) * Nfp + q] * v1[p];
                    b += m->m1d[(f * Nfp + p) * Nfp + q] * v2[p];
                }
                const int n = (int)m->Fmask[q * 3 + f];
                const double nxv = m->nx[(f * Nfp + q) * K + k], nyv = m->ny[(f * Nfp + q) * K + k];
                yk[n] += sJf * a;
                ex[n] -= sJf * nxv * b;
                ey[n] -= sJf * nyv * b;
            }
        }
        for (int i = 0; i < Np; ++i) {
            double s = yk[i];
            for (int j = 0; j < Np; ++j) {
                const double tr = m->rx[j * K + k] * ex[j] + m->ry[j * K + k] * ey[j];
                const double ts = m->sx[j * K + k] * ex[j] + m->sy[j * K + k] * ey[j];
                s += m->Dr[j * Np + i] * tr + m->Ds[j * Np + i] * ts;
            }
            y[k * Np + i] = s;
        }
    }
}
