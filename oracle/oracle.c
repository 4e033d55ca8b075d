/*
 * CPU oracle for the DASH per-timestep force hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into, loaded by, or called from the
 * product library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load the shared object built from it.
 *
 * It restates, from the reference's source, in plain C:
 *   - the periodic wrap            GridGPU.cu:138-161, BoundsGPU.h:128-143
 *   - the cell-binned neighbour predicate (FP32, exactly as compiled by nvcc
 *     with fused multiply-add contraction of dot())
 *                                  GridGPU.cu:326-463, 482-734, cutils_math.h:1566
 *   - the exclusion tag lookup     GridGPU.cu:466-478
 *   - LJ / WCA pair force + energy PairEvaluatorLJ.h:17-60, PairEvaluatorWCA.h:13-38
 *   - Ewald real-space force/energy with the excluded-pair correction
 *                                  ChargeEvaluatorEwald.h:11-64
 *   - the per-atom accumulation    PairEvaluateIso.h:8-207 (virial x0.5, helpers.h:34-41)
 *   - E3B two-body / three-body    EvaluatorE3B.h:67-345, ThreeBodyE3B.h:18-549,
 *                                  parameters FixE3B.cu:515-593
 * Forces/energies are FP64 (the "FP64 CPU oracle"); the neighbour predicate is
 * FP32 because the pair SET must be bit-exact with the FP32 reference.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off, so that the only
 * fused multiply-adds are the explicit fmaf() calls below).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EXCL_MASK (~(3u << 30))

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------------------------------------------------------------------
 * Periodic wrap (GridGPU.cu:138-161): imgs = floorf((x-lo)/L); x -= L*imgs.
 * xs is float4-packed (x,y,z,w); w is left untouched.
 * ------------------------------------------------------------------------- */
void orc_wrap_f32(int n, float *xs4, const float lo[3], const float L[3]) {
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) {
            float x = xs4[4 * i + d];
            float img = floorf((x - lo[d]) / L[d]);
            if (img != 0.0f) {
                float t = L[d] * img; /* exact: img is a small integer */
                xs4[4 * i + d] = x - t;
            }
        }
    }
}

/* FP32 squared distance exactly as the reference's compiled predicate:
 *   distVec = otherPos + shift - pos   (two roundings, shift exact)
 *   dot(distVec,distVec) contracted as fma(z,z,fma(y,y,x*x)). */
static inline float pred_r2(const float *xi, const float *xj, const float sh[3]) {
    float dx = (xj[0] + sh[0]) - xi[0];
    float dy = (xj[1] + sh[1]) - xi[1];
    float dz = (xj[2] + sh[2]) - xi[2];
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

/* exclusion tag of otherId in the list of atom myId (GridGPU.cu:466-478) */
static inline uint32_t excl_tag(const int *excl_start, const uint32_t *excl_ids,
                                int myId, uint32_t otherId) {
    if (!excl_start) return 0;
    for (int e = excl_start[myId]; e < excl_start[myId + 1]; e++) {
        if ((excl_ids[e] & ORC_EXCL_MASK) == otherId) return excl_ids[e] & ~ORC_EXCL_MASK;
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Neighbour list by the reference's cell algorithm (GridGPU.cu:824-1103):
 * cells of width L/ns (ns = floor(L/cut), grid grown by EPSILON), 27-cell
 * stencil with image offset = -floor(cellIdx/ns), predicate pred_r2 < cutsq.
 * Positions must already be wrapped.  Output is in INPUT index order:
 *   counts[i], and nbr[i*maxn + k] = j | tag<<30 (tag = exclusion depth).
 * Returns the largest count seen (entries beyond maxn are dropped).
 * ids[] maps index -> atom id for the exclusion lookup (may be NULL when no
 * exclusions are given).
 * ------------------------------------------------------------------------- */
int orc_nlist_cells(int n, const float *xs4, const float lo[3], const float L[3],
                    float cut, const int *ids, const int *excl_start,
                    const uint32_t *excl_ids, int *counts, uint32_t *nbr, int maxn) {
    int ns[3];
    float ds[3], os[3];
    const float EPS = 0.00001f;
    for (int d = 0; d < 3; d++) {
        ns[d] = (int)((double)L[d] / (double)cut);
        if (ns[d] < 3) return -1; /* reference requires >= 3 cells per side */
        ds[d] = (float)((double)L[d] / ns[d]) + EPS;
        os[d] = lo[d] - EPS;
    }
    int ncell = ns[0] * ns[1] * ns[2];
    int *cellOf = (int *)malloc(sizeof(int) * n);
    int *cstart = (int *)calloc(ncell + 1, sizeof(int));
    int *order = (int *)malloc(sizeof(int) * n);
    int *fill = (int *)calloc(ncell, sizeof(int));
    for (int i = 0; i < n; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) {
            c[d] = (int)((xs4[4 * i + d] - os[d]) / ds[d]);
            if (c[d] < 0) c[d] = 0;
            if (c[d] >= ns[d]) c[d] = ns[d] - 1;
        }
        cellOf[i] = (c[0] * ns[1] + c[1]) * ns[2] + c[2];
        cstart[cellOf[i] + 1]++;
    }
    for (int c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
    for (int i = 0; i < n; i++) order[cstart[cellOf[i]] + fill[cellOf[i]]++] = i;
    const float cutsq = cut * cut;
    int maxc = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : maxc)
    for (int i = 0; i < n; i++) {
        const float *xi = xs4 + 4 * i;
        int ci = cellOf[i];
        int cz = ci % ns[2], cy = (ci / ns[2]) % ns[1], cx = ci / (ns[1] * ns[2]);
        int cnt = 0;
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++)
                for (int oz = -1; oz <= 1; oz++) {
                    int k[3] = {cx + ox, cy + oy, cz + oz};
                    float sh[3];
                    int kw[3];
                    for (int d = 0; d < 3; d++) {
                        int off = (int)(-floorf((float)k[d] / ns[d]));
                        kw[d] = k[d] + ns[d] * off;
                        sh[d] = (float)(-off) * L[d];
                    }
                    int c = (kw[0] * ns[1] + kw[1]) * ns[2] + kw[2];
                    for (int p = cstart[c]; p < cstart[c + 1]; p++) {
                        int j = order[p];
                        if (j == i) continue;
                        if (pred_r2(xi, xs4 + 4 * j, sh) < cutsq) {
                            if (cnt < maxn) {
                                uint32_t tag = ids ? excl_tag(excl_start, excl_ids, ids[i], (uint32_t)ids[j]) : 0;
                                nbr[(size_t)i * maxn + cnt] = (uint32_t)j | tag;
                            }
                            cnt++;
                        }
                    }
                }
        counts[i] = cnt;
        if (cnt > maxc) maxc = cnt;
    }
    free(cellOf);
    free(cstart);
    free(order);
    free(fill);
    return maxc;
}

/* Brute-force cross-check of the same predicate with the minimum-image shift
 * chosen per dimension; O(N^2), small systems only. */
int orc_nlist_brute(int n, const float *xs4, const float L[3], float cut,
                    int *counts, uint32_t *nbr, int maxn) {
    const float cutsq = cut * cut;
    int maxc = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : maxc)
    for (int i = 0; i < n; i++) {
        int cnt = 0;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            float sh[3];
            for (int d = 0; d < 3; d++) {
                double dx = (double)xs4[4 * j + d] - (double)xs4[4 * i + d];
                double img = -rint(dx / (double)L[d]);
                sh[d] = (float)img * L[d];
            }
            if (pred_r2(xs4 + 4 * i, xs4 + 4 * j, sh) < cutsq) {
                if (cnt < maxn) nbr[(size_t)i * maxn + cnt] = (uint32_t)j;
                cnt++;
            }
        }
        counts[i] = cnt;
        if (cnt > maxc) maxc = cnt;
    }
    return maxc;
}

/* ---------------------------------------------------------------------------
 * Pair forces over a neighbour list (PairEvaluateIso.h:8-207), FP64.
 *   lj_kind: 0 none, 1 LJ/cut (PairEvaluatorLJ.h), 2 WCA (PairEvaluatorWCA.h)
 *   params per type pair (row-major ntypes x ntypes): rc2, eps24, sig6
 *   coulomb: if qrc > 0, Ewald real space (ChargeEvaluatorEwald.h) with
 *            qqr_to_eng, alpha; exclusion multiplier from the list tag.
 * Outputs (each may be NULL): f[3n], virial[6n] (xx,yy,zz,xy,xz,yz, x0.5),
 * energy[n] (per-atom, half-counted as the reference).
 * ------------------------------------------------------------------------- */
void orc_pair_forces(int n, const double *x, const int *type, const double *q,
                     int ntypes, const double *rc2, const double *eps24, const double *sig6,
                     int lj_kind, double qrc, double alpha, double qqr_to_eng,
                     const double L[3], const int *counts, const uint32_t *nbr, int maxn,
                     const double coef[4], double *f, double *virial, double *energy) {
    const double qrc2 = qrc * qrc;
    const double two_over_sqrtpi = 2.0 * 0.5641895835477563;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        double fx = 0, fy = 0, fz = 0, e = 0;
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < counts[i]; k++) {
            uint32_t raw = nbr[(size_t)i * maxn + k];
            int j = (int)(raw & ORC_EXCL_MASK);
            double mult = coef[raw >> 30];
            double dr[3];
            for (int d = 0; d < 3; d++) {
                double t = x[3 * i + d] - x[3 * j + d];
                dr[d] = t - L[d] * rint(t / L[d]);
            }
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            double fs = 0.0;
            int any = 0;
            int tp = type[i] * ntypes + type[j];
            if (lj_kind && r2 < rc2[tp]) {
                any = 1;
                if (mult != 0.0) {
                    double p1 = eps24[tp] * 2.0 * sig6[tp] * sig6[tp];
                    double p2 = eps24[tp] * sig6[tp];
                    double r2inv = 1.0 / r2;
                    double r6inv = r2inv * r2inv * r2inv;
                    fs += r6inv * r2inv * (p1 * r6inv - p2) * mult;
                    double eps = eps24[tp] / 24.0;
                    double s6r6 = sig6[tp] * r6inv;
                    if (lj_kind == 1) {
                        double rc6 = rc2[tp] * rc2[tp] * rc2[tp];
                        double s6rc6 = sig6[tp] / rc6;
                        double off = s6rc6 * (s6rc6 - 1.0);
                        e += 0.5 * 4.0 * eps * (s6r6 * (s6r6 - 1.0) - off) * mult;
                    } else {
                        e += 0.5 * (4.0 * eps * s6r6 * (s6r6 - 1.0) + eps) * mult;
                    }
                }
            }
            if (qrc > 0.0 && r2 < qrc2) {
                any = 1;
                double rr2 = r2 < 1e-10 ? 1e-10 : r2;
                double r2inv = 1.0 / rr2;
                double rinv = sqrt(r2inv);
                double len = sqrt(rr2);
                double qq = qqr_to_eng * q[i] * q[j];
                double s = qq * (erfc(alpha * len) * rinv + two_over_sqrtpi * alpha * exp(-alpha * alpha * rr2));
                if (mult < 1.0) s -= (1.0 - mult) * qq * rinv;
                fs += s * r2inv;
                double eng = qq * rinv * erfc(alpha * len);
                if (mult < 1.0) eng -= (1.0 - mult) * qq * rinv;
                e += 0.5 * eng;
            }
            if (any) {
                double F[3] = {dr[0] * fs, dr[1] * fs, dr[2] * fs};
                fx += F[0];
                fy += F[1];
                fz += F[2];
                v[0] += F[0] * dr[0];
                v[1] += F[1] * dr[1];
                v[2] += F[2] * dr[2];
                v[3] += F[0] * dr[1];
                v[4] += F[0] * dr[2];
                v[5] += F[1] * dr[2];
            }
        }
        if (f) {
            f[3 * i] = fx;
            f[3 * i + 1] = fy;
            f[3 * i + 2] = fz;
        }
        if (virial)
            for (int c = 0; c < 6; c++) virial[6 * i + c] = 0.5 * v[c];
        if (energy) energy[i] = e;
    }
}

/* ---------------------------------------------------------------------------
 * The other pair styles of compute_force_iso, FP64, on a list as above.
 *   params: np x ntypes x ntypes processed tables in the reference's
 *     paramOrder; lj_kind 1 LJ/cut {rc2, 24eps, sig6} (PairEvaluatorLJ.h:17-60),
 *     3 force-shifted LJ {rc2, 24eps, sig6, F(rc)} (PairEvaluatorLJFS.h:15-57),
 *     4 CHARMM {rc2, 24eps, sig6, 24eps14, sig14^6} (PairEvaluatorCHARMM.h:7-44,
 *     a pair whose multiplier equals coef[3] takes the 1-4 parameters),
 *     5 TICG {rc2, C} (PairEvaluatorTICG.h:9-52), 0 none.
 *   ck: 0 no charges, 1 Ewald real space (ChargeEvaluatorEwald.h:11-64),
 *     2 damped shifted force (ChargeEvaluatorDSF.h:13-47) with
 *     dsf = {2 alpha/sqrt(pi), shift, erfc(alpha rc)/rc, rc}.
 * Outputs as orc_pair_forces.
 * ------------------------------------------------------------------------- */
void orc_pair_forces_styles(int n, const double *x, const int *type, const double *q, int ntypes,
                            const double *params, int np, int lj_kind, int ck, double qrc, double alpha,
                            double qqr_to_eng, const double *dsf, const double L[3], const int *counts,
                            const uint32_t *nbr, int maxn, const double coef[4], double *f, double *virial,
                            double *energy) {
    const double qrc2 = qrc * qrc;
    const double two_over_sqrtpi = 2.0 * 0.5641895835477563;
    const int nt2 = ntypes * ntypes;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        double fx = 0, fy = 0, fz = 0, e = 0;
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < counts[i]; k++) {
            uint32_t raw = nbr[(size_t)i * maxn + k];
            int j = (int)(raw & ORC_EXCL_MASK);
            double mult = coef[raw >> 30];
            double dr[3];
            for (int d = 0; d < 3; d++) {
                double t = x[3 * i + d] - x[3 * j + d];
                dr[d] = t - L[d] * rint(t / L[d]);
            }
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            double fs = 0.0;
            int any = 0;
            int tp = type[i] * ntypes + type[j];
            (void)np;
            if (lj_kind && r2 < params[tp]) {
                const double rc2 = params[tp];
                any = 1;
                if (mult != 0.0) {
                    if (lj_kind == 5) {
                        const double C = params[nt2 + tp];
                        if (r2 != 0.0) fs += -C * 1.5 / sqrt(rc2 * r2) * (r2 / rc2 - 1.0) * mult;
                        const double xr = sqrt(r2 / rc2);
                        e += 0.5 * C * (0.5 * (xr - 1.0) * (xr - 1.0) * (xr + 2.0)) * mult;
                    } else {
                        double eps24 = params[nt2 + tp], sig6 = params[2 * nt2 + tp];
                        if (lj_kind == 4 && mult == coef[3]) {
                            eps24 = params[3 * nt2 + tp];
                            sig6 = params[4 * nt2 + tp];
                        }
                        const double p1 = eps24 * 2.0 * sig6 * sig6, p2 = eps24 * sig6;
                        const double r2inv = 1.0 / r2, r6inv = r2inv * r2inv * r2inv;
                        double s = r6inv * r2inv * (p1 * r6inv - p2);
                        if (lj_kind == 3) s -= params[3 * nt2 + tp] / sqrt(r2);
                        fs += s * mult;
                        const double eps = eps24 / 24.0, s6r6 = sig6 * r6inv;
                        const double rc6 = rc2 * rc2 * rc2, s6rc6 = sig6 / rc6;
                        double u = 4.0 * eps * (s6r6 * (s6r6 - 1.0) - s6rc6 * (s6rc6 - 1.0));
                        /* U(r) - U(rc) + F(rc) (r - rc): the force-consistent form the
                           reference documents (PairEvaluatorLJFS.h:41-44); its code adds
                           F(rc) (rc - r) */
                        if (lj_kind == 3) u += params[3 * nt2 + tp] * (sqrt(r2) - sqrt(rc2));
                        e += 0.5 * u * mult;
                    }
                }
            }
            if (ck == 1 && r2 < qrc2) {
                any = 1;
                double rr2 = r2 < 1e-10 ? 1e-10 : r2;
                double r2inv = 1.0 / rr2, rinv = sqrt(r2inv), len = sqrt(rr2);
                double qq = qqr_to_eng * q[i] * q[j];
                double s = qq * (erfc(alpha * len) * rinv + two_over_sqrtpi * alpha * exp(-alpha * alpha * rr2));
                if (mult < 1.0) s -= (1.0 - mult) * qq * rinv;
                fs += s * r2inv;
                double eng = qq * rinv * erfc(alpha * len);
                if (mult < 1.0) eng -= (1.0 - mult) * qq * rinv;
                e += 0.5 * eng;
            }
            if (ck == 2 && r2 < qrc2) {
                any = 1;
                double r2inv = 1.0 / r2, rinv = sqrt(r2inv), len = sqrt(r2);
                double qq = qqr_to_eng * q[i] * q[j];
                fs += qq * (erfc(alpha * len) * r2inv + dsf[0] * exp(-alpha * alpha * r2) * rinv - dsf[1]) * rinv * mult;
                e += 0.5 * qq * (erfc(alpha * len) * rinv - dsf[2] + dsf[1] * (len - dsf[3])) * mult;
            }
            if (any) {
                double F[3] = {dr[0] * fs, dr[1] * fs, dr[2] * fs};
                fx += F[0];
                fy += F[1];
                fz += F[2];
                v[0] += F[0] * dr[0];
                v[1] += F[1] * dr[1];
                v[2] += F[2] * dr[2];
                v[3] += F[0] * dr[1];
                v[4] += F[0] * dr[2];
                v[5] += F[1] * dr[2];
            }
        }
        if (f) {
            f[3 * i] = fx;
            f[3 * i + 1] = fy;
            f[3 * i + 2] = fz;
        }
        if (virial)
            for (int c = 0; c < 6; c++) virial[6 * i + c] = 0.5 * v[c];
        if (energy) energy[i] = e;
    }
}

/* ---------------------------------------------------------------------------
 * E3B (EvaluatorE3B.h, ThreeBodyE3B.h).  Molecules are (O, H1, H2, M) atom
 * indices into x.  All O-O pairs with r < r2b_cut (the reference's molecule
 * list radius rf + 1 A) get the two-body term; pairs with r <= rmax3 get the
 * three-body terms.  The list is brute force over molecule pairs (O(M^2)).
 * prm = {rs, rf, E2, Ea, Eb, Ec, k2, k3, r2b_cut, rmax3}
 * Outputs f[3*natoms] (added to), energy[natoms] (added to), may be NULL.
 * ------------------------------------------------------------------------- */
typedef struct {
    double rs, rf, E2, Ea, Eb, Ec, k2, k3;
} e3b_par;

static inline double e3b_sw(const e3b_par *p, double r) {
    if (r <= p->rs) return 1.0;
    if (r > p->rf) return 0.0;
    double d = p->rf - p->rs;
    double v = (p->rf - r);
    v *= v;
    v *= (p->rf + 2.0 * r - 3.0 * p->rs) / (d * d * d);
    return v;
}
static inline double e3b_dsw(const e3b_par *p, double r) {
    if (r <= p->rs || r > p->rf) return 0.0;
    double d = p->rf - p->rs;
    return 6.0 * (p->rf - r) * (p->rs - r) / (d * d * d);
}
static inline double e3b_e(const e3b_par *p, double r) { return e3b_sw(p, r) * exp(-p->k3 * r); }
/* threeBodyForce: vector along dr (points from O to H) */
static inline void e3b_f(const e3b_par *p, const double dr[3], double r, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    if (r <= p->rf) {
        double es = exp(-p->k3 * r);
        double s = p->k3 * es / r;
        if (r > p->rs) {
            s *= e3b_sw(p, r);
            s -= es * e3b_dsw(p, r) / r;
        }
        out[0] = dr[0] * s;
        out[1] = dr[1] * s;
        out[2] = dr[2] * s;
    }
}

static inline void mimg(const double *a, const double *b, const double L[3], double out[3]) {
    for (int d = 0; d < 3; d++) {
        double t = a[d] - b[d];
        out[d] = t - L[d] * rint(t / L[d]);
    }
}
static inline double len3(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

/* per-pair geometry for molecules (1=a, 2=b) as ThreeBodyE3B.h:128-176 */
typedef struct {
    double es[4];     /* e_b2a1, e_c2a1, e_b1a2, e_c1a2 */
    double fv[4][3];  /* forces_b2a1, c2a1, b1a2, c1a2 */
} e3b_pair;

static void e3b_pair_geom(const e3b_par *p, const double *x, const int *ma, const int *mb,
                          const double L[3], e3b_pair *out) {
    const double *a1 = x + 3 * ma[0], *b1 = x + 3 * ma[1], *c1 = x + 3 * ma[2];
    const double *a2 = x + 3 * mb[0], *b2 = x + 3 * mb[1], *c2 = x + 3 * mb[2];
    double d[4][3];
    mimg(b2, a1, L, d[0]);
    mimg(c2, a1, L, d[1]);
    mimg(b1, a2, L, d[2]);
    mimg(c1, a2, L, d[3]);
    for (int k = 0; k < 4; k++) {
        double r = len3(d[k]);
        out->es[k] = e3b_e(p, r);
        e3b_f(p, d[k], r, out->fv[k]);
    }
}

/* EvaluatorE3B::threeBodyPairForce (EvaluatorE3B.h:145-249) with totals
 * T1 (this molecule) and T2 (other).  Adds to f1[3][3] (a1,b1,c1) and
 * f2[3][3] (a2,b2,c2). */
static void e3b_pair_force(const e3b_par *p, const e3b_pair *g, const double T1[3],
                           const double T2[3], double f1[3][3], double f2[3][3]) {
    const double *e = g->es;
    double sc;
#define ADDF(dst, src, s) \
    do { (dst)[0] += (s) * (src)[0]; (dst)[1] += (s) * (src)[1]; (dst)[2] += (s) * (src)[2]; } while (0)
    /* type A */
    sc = p->Ea * (T2[1] - e[0]);
    ADDF(f1[0], g->fv[1], -sc); ADDF(f2[2], g->fv[1], sc);
    sc = p->Ea * (T1[1] - e[2]);
    ADDF(f2[0], g->fv[3], -sc); ADDF(f1[2], g->fv[3], sc);
    sc = p->Ea * (T2[2] - e[1]);
    ADDF(f1[0], g->fv[0], -sc); ADDF(f2[1], g->fv[0], sc);
    sc = p->Ea * (T1[2] - e[3]);
    ADDF(f2[0], g->fv[2], -sc); ADDF(f1[1], g->fv[2], sc);
    /* type B */
    sc = p->Eb * (T2[0] + T1[1] + T1[2] - 2.0 * (e[2] + e[3]));
    ADDF(f1[0], g->fv[0], -sc); ADDF(f2[1], g->fv[0], sc);
    ADDF(f1[0], g->fv[1], -sc); ADDF(f2[2], g->fv[1], sc);
    sc = p->Eb * (T1[0] + T2[1] + T2[2] - 2.0 * (e[0] + e[1]));
    ADDF(f2[0], g->fv[2], -sc); ADDF(f1[1], g->fv[2], sc);
    ADDF(f2[0], g->fv[3], -sc); ADDF(f1[2], g->fv[3], sc);
    /* type C */
    sc = p->Ec * (T1[0] - e[1] - e[0]);
    ADDF(f1[0], g->fv[0], -sc); ADDF(f2[1], g->fv[0], sc);
    ADDF(f1[0], g->fv[1], -sc); ADDF(f2[2], g->fv[1], sc);
    sc = p->Ec * (T2[0] - e[2] - e[3]);
    ADDF(f2[0], g->fv[2], -sc); ADDF(f1[1], g->fv[2], sc);
    ADDF(f2[0], g->fv[3], -sc); ADDF(f1[2], g->fv[3], sc);
#undef ADDF
}

/* EvaluatorE3B::threeBodyPairEnergy (EvaluatorE3B.h:251-345): total energy of
 * one unordered pair (sum of the per-atom quarter terms). */
static double e3b_pair_energy(const e3b_par *p, const double *e, const double T1[3], const double T2[3]) {
    double s = 0.0, sc;
    sc = p->Ea * (T2[1] - e[0]); s += 0.25 * sc * e[1] * 2.0;
    sc = p->Ea * (T1[1] - e[2]); s += 0.25 * sc * e[3] * 2.0;
    sc = p->Ea * (T2[2] - e[1]); s += 0.25 * sc * e[0] * 2.0;
    sc = p->Ea * (T1[2] - e[3]); s += 0.25 * sc * e[2] * 2.0;
    sc = p->Eb * (T2[0] + T1[1] + T1[2] - 2.0 * (e[2] + e[3]));
    s += 0.25 * sc * (e[0] + e[1]) * 2.0;
    sc = p->Eb * (T1[0] + T2[1] + T2[2] - 2.0 * (e[0] + e[1]));
    s += 0.25 * sc * (e[2] + e[3]) * 2.0;
    sc = p->Ec * (T1[0] - e[1] - e[0]);
    s += 0.25 * sc * (e[0] + e[1]) * 2.0;
    sc = p->Ec * (T2[0] - e[2] - e[3]);
    s += 0.25 * sc * (e[2] + e[3]) * 2.0;
    return s;
}

/* returns number of three-body pairs evaluated */
/* e3b_pair_force's forces are central O-H pair forces sc * fv[k] along
 * d[k] (H minus O, minimum image); their virial is sum_k S_k fv[k] (x) d[k]
 * with S_k the sum of the coefficients that multiply fv[k] there.  Adds to
 * vir[6] (xx yy zz xy xz yz, computeVirial's order, helpers.h:34-41). */
static void e3b_pair_virial(const e3b_par *p, const e3b_pair *g, const double d[4][3], const double T1[3],
                            const double T2[3], double vir[6]) {
    const double *e = g->es;
    const double B1 = p->Eb * (T2[0] + T1[1] + T1[2] - 2.0 * (e[2] + e[3]));
    const double B2 = p->Eb * (T1[0] + T2[1] + T2[2] - 2.0 * (e[0] + e[1]));
    const double C1 = p->Ec * (T1[0] - e[1] - e[0]);
    const double C2 = p->Ec * (T2[0] - e[2] - e[3]);
    const double S[4] = {p->Ea * (T2[2] - e[1]) + B1 + C1, p->Ea * (T2[1] - e[0]) + B1 + C1,
                         p->Ea * (T1[2] - e[3]) + B2 + C2, p->Ea * (T1[1] - e[2]) + B2 + C2};
    for (int k = 0; k < 4; k++) {
        const double *fv = g->fv[k], *dk = d[k];
        vir[0] += S[k] * fv[0] * dk[0];
        vir[1] += S[k] * fv[1] * dk[1];
        vir[2] += S[k] * fv[2] * dk[2];
        vir[3] += S[k] * fv[0] * dk[1];
        vir[4] += S[k] * fv[0] * dk[2];
        vir[5] += S[k] * fv[1] * dk[2];
    }
}

/* vir (may be NULL): total virial, two-body as the reference (0.5 F (x) dr
 * per ordered pair, ThreeBodyE3B.h:129, 222-245) plus the three-body pair
 * forces (which the reference leaves out, ThreeBodyE3B.h:449-451) */
int orc_e3b(int nmol, const int *mol, const double *x, const double L[3], const double *prm,
            double *f, double *energy_total, double *vir) {
    e3b_par p = {prm[0], prm[1], prm[2], prm[3], prm[4], prm[5], prm[6], prm[7]};
    const double r2b = prm[8], rmax3 = prm[9];
    double *T = (double *)calloc((size_t)3 * nmol, sizeof(double));
    double e2 = 0.0, e3 = 0.0;
    double v2[6] = {0, 0, 0, 0, 0, 0};
    int npairs = 0;
    /* pass 1: totals (ThreeBodyE3B.h:170-211) and the two-body force */
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : e2, v2[:6])
    for (int a = 0; a < nmol; a++) {
        const int *ma = mol + 4 * a;
        double fo[3] = {0, 0, 0};
        for (int b = 0; b < nmol; b++) {
            if (b == a) continue;
            const int *mb = mol + 4 * b;
            double d[3];
            mimg(x + 3 * ma[0], x + 3 * mb[0], L, d);
            double r = len3(d);
            if (r >= r2b) continue;
            double s = p.k2 * p.E2 * exp(-p.k2 * r) / r;
            fo[0] += d[0] * s;
            fo[1] += d[1] * s;
            fo[2] += d[2] * s;
            v2[0] += 0.5 * s * d[0] * d[0];
            v2[1] += 0.5 * s * d[1] * d[1];
            v2[2] += 0.5 * s * d[2] * d[2];
            v2[3] += 0.5 * s * d[0] * d[1];
            v2[4] += 0.5 * s * d[0] * d[2];
            v2[5] += 0.5 * s * d[1] * d[2];
            e2 += 0.5 * p.E2 * exp(-p.k2 * r);
            if (r <= rmax3) {
                e3b_pair g;
                e3b_pair_geom(&p, x, ma, mb, L, &g);
                T[3 * a + 0] += g.es[0] + g.es[1];
                T[3 * a + 1] += g.es[2];
                T[3 * a + 2] += g.es[3];
            }
        }
        if (f) {
            f[3 * ma[0]] += fo[0];
            f[3 * ma[0] + 1] += fo[1];
            f[3 * ma[0] + 2] += fo[2];
        }
    }
    /* pass 2: pair forces, each unordered pair once with (1=a<2=b) as the
     * reference (ThreeBodyE3B.h:185, 368-437); serial to keep the sum order */
    for (int a = 0; a < nmol; a++) {
        const int *ma = mol + 4 * a;
        for (int b = a + 1; b < nmol; b++) {
            const int *mb = mol + 4 * b;
            double d[3];
            mimg(x + 3 * ma[0], x + 3 * mb[0], L, d);
            double r = len3(d);
            if (!(r < r2b && r <= rmax3)) continue;
            e3b_pair g;
            e3b_pair_geom(&p, x, ma, mb, L, &g);
            double f1[3][3] = {{0}}, f2[3][3] = {{0}};
            e3b_pair_force(&p, &g, T + 3 * a, T + 3 * b, f1, f2);
            if (vir) {
                double dd[4][3];
                mimg(x + 3 * mb[1], x + 3 * ma[0], L, dd[0]);
                mimg(x + 3 * mb[2], x + 3 * ma[0], L, dd[1]);
                mimg(x + 3 * ma[1], x + 3 * mb[0], L, dd[2]);
                mimg(x + 3 * ma[2], x + 3 * mb[0], L, dd[3]);
                e3b_pair_virial(&p, &g, (const double(*)[3])dd, T + 3 * a, T + 3 * b, vir);
            }
            if (f) {
                for (int s = 0; s < 3; s++)
                    for (int c = 0; c < 3; c++) {
                        f[3 * ma[s] + c] += f1[s][c];
                        f[3 * mb[s] + c] += f2[s][c];
                    }
            }
            e3 += e3b_pair_energy(&p, g.es, T + 3 * a, T + 3 * b);
            npairs++;
        }
    }
    if (energy_total) {
        energy_total[0] = e2;
        energy_total[1] = e3;
    }
    if (vir)
        for (int c = 0; c < 6; c++) vir[c] += v2[c];
    free(T);
    return npairs;
}

/* Host-callable single-pair helpers used to pin the oracle's per-pair maths
 * against the reference's own host/device functors and known answers. */
void orc_lj_force_single(double sigma, double eps, double rcut, const double dr[3], double out[3]) {
    double sig6 = pow(sigma, 6.0), eps24 = 24.0 * eps;
    double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
    out[0] = out[1] = out[2] = 0.0;
    if (r2 >= rcut * rcut) return;
    double p1 = eps24 * 2.0 * sig6 * sig6, p2 = eps24 * sig6;
    double r2inv = 1.0 / r2, r6inv = r2inv * r2inv * r2inv;
    double s = r6inv * r2inv * (p1 * r6inv - p2);
    out[0] = dr[0] * s;
    out[1] = dr[1] * s;
    out[2] = dr[2] * s;
}

void orc_e3b_single(const double *prm, double r, double out[4]) {
    /* switching, dswitch, threeBodyPairEnergy, threeBodyForce scalar */
    e3b_par p = {prm[0], prm[1], prm[2], prm[3], prm[4], prm[5], prm[6], prm[7]};
    out[0] = e3b_sw(&p, r);
    out[1] = e3b_dsw(&p, r);
    out[2] = e3b_e(&p, r);
    double dr[3] = {r, 0, 0}, fv[3];
    e3b_f(&p, dr, r, fv);
    out[3] = fv[0];
}
