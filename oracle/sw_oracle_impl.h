/*
 * TEST INFRASTRUCTURE ONLY — never linked into the product.
 *
 * Body of the CPU oracle for soft Smith–Waterman (linear and affine gaps).
 * sw_oracle.c includes this file twice: once with REAL=float (a restatement
 * that follows the reference CPU kernels operation by operation, so it can be
 * compared bit-for-bit with them) and once with REAL=double (the FP64 truth
 * that errors are reported against).
 *
 * Every function states which reference routine it restates; paths are inside
 * megure-labs/orihime.
 *
 * Semantics shared by all routines (src/common/numerics.h:29-127):
 *   NEG_BIG = -1e30 stands for "no path"; an LSE whose max is <= NEG_BIG is
 *   NEG_BIG; exp arguments below -88 give 0 and are clamped to 88 above;
 *   sums of exponentials are Kahan-compensated.
 * DP indices are 1-based: cell (i,j) uses score s[i-1][j-1]; row 0 / column 0
 * are boundary cells (only M[0,0] = 0 is a live value).
 */

#ifndef REAL
#error "define REAL before including sw_oracle_impl.h"
#endif

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* ---- scalar helpers ---------------------------------------------------- */

static REAL FN(clip_exp)(REAL x) {
    if (x < (REAL)-88.0) return (REAL)0;
    if (x > (REAL)88.0) x = (REAL)88.0;
    return EXPF(x);
}

typedef struct { REAL s, c; } FN(ksum_t);

static void FN(kadd)(FN(ksum_t) *k, REAL v) {
    REAL y = v - k->c;
    REAL t = k->s + y;
    k->c = (t - k->s) - y;
    k->s = t;
}

static REAL FN(vmax)(const REAL *v, int n) {
    REAL m = v[0];
    for (int q = 1; q < n; ++q) if (v[q] > m) m = v[q];
    return m;
}

/* T*log(sum exp(v/T)) over n terms (numerics.h:75-127). */
static REAL FN(tlse)(const REAL *v, int n, REAL T) {
    REAL m = FN(vmax)(v, n);
    if (m <= (REAL)NEG_BIG) return (REAL)NEG_BIG;
    FN(ksum_t) k = {0, 0};
    for (int q = 0; q < n; ++q) FN(kadd)(&k, FN(clip_exp)((v[q] - m) / T));
    return m + T * LOGF(k.s);
}

/* Normalised softmax weights, zero for NEG_BIG terms
 * (src/sw_affine/kernels_cpu.cpp:56-88, src/sw/kernels_cpu.cpp:42-63). */
static void FN(tsoftmax)(const REAL *v, int n, REAL T, REAL *w) {
    REAL m = FN(vmax)(v, n);
    if (m <= (REAL)NEG_BIG) { for (int q = 0; q < n; ++q) w[q] = 0; return; }
    FN(ksum_t) k = {0, 0};
    for (int q = 0; q < n; ++q) {
        if (v[q] > (REAL)NEG_BIG) { w[q] = FN(clip_exp)((v[q] - m) / T); FN(kadd)(&k, w[q]); }
        else w[q] = 0;
    }
    if (k.s > 0) for (int q = 0; q < n; ++q) w[q] /= k.s;
}

/* exp(min((a - S)/T, 0)), or 0 for a dead cell (kernels_cpu.cpp:43-52). */
static REAL FN(end_weight)(REAL a, REAL S, REAL T) {
    if (a <= (REAL)NEG_BIG) return 0;
    REAL lp = (a - S) / T;
    if (lp > 0) lp = 0;
    return FN(clip_exp)(lp);
}

static int FN(live)(REAL b) { return !(isinf(b) || isnan(b) || b == 0); }

/* ---- affine model ------------------------------------------------------ */

/* Tables of one pair: plane 0 = M, 1 = I, 2 = D, each (L1+1) x (L2+1). */
typedef struct {
    int L1, L2, ld;          /* ld = row pitch of the score slab */
    const REAL *s;
    REAL go, ge, T;
    size_t plane, cols;
    REAL *a;                 /* 3 planes */
} FN(aff_t);

#define AIX(c, st, i, j) ((size_t)(st) * (c)->plane + (size_t)(i) * (c)->cols + (size_t)(j))
#define SC(c, i, j) ((c)->s[(size_t)((i) - 1) * (c)->ld + (size_t)((j) - 1)])

/* The three candidate vectors of cell (i,j): M (diag M,I,D + s, sky s),
 * I (up M + go, up I + ge), D (left M + go, left D + ge). */
static void FN(aff_cands)(const FN(aff_t) *c, const REAL *tab, int i, int j,
                          REAL vm[4], REAL vi[2], REAL vd[2]) {
    REAL s = SC(c, i, j);
    int dg = (i > 1 && j > 1);
    vm[0] = dg ? tab[AIX(c, 0, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    vm[1] = dg ? tab[AIX(c, 1, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    vm[2] = dg ? tab[AIX(c, 2, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    vm[3] = s;
    vi[0] = (i > 1) ? tab[AIX(c, 0, i - 1, j)] + c->go : (REAL)NEG_BIG;
    vi[1] = (i > 1) ? tab[AIX(c, 1, i - 1, j)] + c->ge : (REAL)NEG_BIG;
    vd[0] = (j > 1) ? tab[AIX(c, 0, i, j - 1)] + c->go : (REAL)NEG_BIG;
    vd[1] = (j > 1) ? tab[AIX(c, 2, i, j - 1)] + c->ge : (REAL)NEG_BIG;
}

/* Forward tables and log-partition (src/sw_affine/kernels_cpu.cpp:94-195).
 * Cells are visited row-major; every cell reads only cells with smaller
 * i+j, so the values equal the reference's anti-diagonal order bit for bit. */
static REAL FN(aff_forward)(FN(aff_t) *c) {
    size_t n = 3 * c->plane;
    for (size_t q = 0; q < n; ++q) c->a[q] = (REAL)NEG_BIG;
    c->a[0] = 0;
    REAL vm[4], vi[2], vd[2];
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            FN(aff_cands)(c, c->a, i, j, vm, vi, vd);
            c->a[AIX(c, 0, i, j)] = FN(tlse)(vm, 4, c->T);
            c->a[AIX(c, 1, i, j)] = FN(tlse)(vi, 2, c->T);
            c->a[AIX(c, 2, i, j)] = FN(tlse)(vd, 2, c->T);
        }
    REAL m = (REAL)NEG_BIG;
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st) {
                REAL v = c->a[AIX(c, st, i, j)];
                if (v > m) m = v;
            }
    FN(ksum_t) k = {0, 0};
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st) {
                REAL v = c->a[AIX(c, st, i, j)];
                if (v > (REAL)NEG_BIG) FN(kadd)(&k, FN(clip_exp)((v - m) / c->T));
            }
    return m + c->T * LOGF(k.s);
}

/* Adjoint pass (src/sw_affine/kernels_cpu.cpp:201-356): beta starts at the
 * clamped end weight of every state, then flows to predecessors in reverse
 * anti-diagonal order (i ascending within a diagonal; per cell M, then I,
 * then D).  post is the pair's padded [L1max x ld] slab, zeroed here.
 * g[0]=dS/dgo, g[1]=dS/dge, g[2]=dS/dT. */
static void FN(aff_adjoint)(const FN(aff_t) *c, REAL S, REAL *be, REAL *post,
                            int L1max, REAL g[3]) {
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < nsc; ++q) post[q] = 0;
    size_t n = 3 * c->plane;
    for (size_t q = 0; q < n; ++q) be[q] = 0;
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st) {
                REAL lp = (c->a[AIX(c, st, i, j)] - S) / c->T;
                if (lp > 0) lp = 0;
                be[AIX(c, st, i, j)] = FN(clip_exp)(lp);
            }
    REAL gopen = 0, gext = 0;
    REAL vm[4], vi[2], vd[2], wm[4], wi[2], wd[2];
    for (int k = c->L1 + c->L2; k >= 2; --k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            FN(aff_cands)(c, c->a, i, j, vm, vi, vd);
            REAL bm = be[AIX(c, 0, i, j)];
            if (FN(live)(bm)) {
                FN(tsoftmax)(vm, 4, c->T, wm);
                post[(size_t)(i - 1) * c->ld + (j - 1)] += bm * (wm[0] + wm[1] + wm[2] + wm[3]);
                if (i > 1 && j > 1)
                    for (int st = 0; st < 3; ++st)
                        if (wm[st] > 0) be[AIX(c, st, i - 1, j - 1)] += bm * wm[st];
            }
            REAL bi = be[AIX(c, 1, i, j)];
            if (FN(live)(bi)) {
                FN(tsoftmax)(vi, 2, c->T, wi);
                if (i > 1) {
                    if (wi[0] > 0) { be[AIX(c, 0, i - 1, j)] += bi * wi[0]; gopen += bi * wi[0]; }
                    if (wi[1] > 0) { be[AIX(c, 1, i - 1, j)] += bi * wi[1]; gext += bi * wi[1]; }
                }
            }
            REAL bd = be[AIX(c, 2, i, j)];
            if (FN(live)(bd)) {
                FN(tsoftmax)(vd, 2, c->T, wd);
                if (j > 1) {
                    if (wd[0] > 0) { be[AIX(c, 0, i, j - 1)] += bd * wd[0]; gopen += bd * wd[0]; }
                    if (wd[1] > 0) { be[AIX(c, 2, i, j - 1)] += bd * wd[1]; gext += bd * wd[1]; }
                }
            }
        }
    }
    /* Expected match score over the whole padded slab, as the reference does. */
    FN(ksum_t) ms = {0, 0};
    for (int r = 0; r < L1max; ++r)
        for (int q = 0; q < c->ld; ++q) {
            size_t o = (size_t)r * c->ld + q;
            FN(kadd)(&ms, post[o] * c->s[o]);
        }
    REAL gap_cost = gopen * c->go + gext * c->ge;
    REAL total = ms.s + gap_cost;
    g[0] = gopen;
    g[1] = gext;
    g[2] = (S - total) / c->T;
}

/* Hessian-vector product d(post)/d(scores) . V
 * (src/sw_affine/kernels_cpu.cpp:362-631): tangent forward of alpha along V,
 * tangent of the partition, then beta and its tangent pushed backwards. */
static void FN(aff_hvp)(const FN(aff_t) *c, REAL S, const REAL *V, REAL *da,
                        REAL *be, REAL *dbe, REAL *H, int L1max) {
    size_t n = 3 * c->plane;
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < n; ++q) { da[q] = 0; dbe[q] = 0; be[q] = 0; }
    for (size_t q = 0; q < nsc; ++q) H[q] = 0;
    REAL vm[4], vi[2], vd[2], wm[4], wi[2], wd[2];
#define VV(i, j) V[(size_t)((i) - 1) * c->ld + (size_t)((j) - 1)]
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            REAL v = VV(i, j);
            int dg = (i > 1 && j > 1);
            FN(aff_cands)(c, c->a, i, j, vm, vi, vd);
            FN(tsoftmax)(vm, 4, c->T, wm);
            REAL t0 = dg ? da[AIX(c, 0, i - 1, j - 1)] + v : 0;
            REAL t1 = dg ? da[AIX(c, 1, i - 1, j - 1)] + v : 0;
            REAL t2 = dg ? da[AIX(c, 2, i - 1, j - 1)] + v : 0;
            da[AIX(c, 0, i, j)] = wm[0] * t0 + wm[1] * t1 + wm[2] * t2 + wm[3] * v;
            FN(tsoftmax)(vi, 2, c->T, wi);
            REAL u0 = (i > 1) ? da[AIX(c, 0, i - 1, j)] : 0;
            REAL u1 = (i > 1) ? da[AIX(c, 1, i - 1, j)] : 0;
            da[AIX(c, 1, i, j)] = wi[0] * u0 + wi[1] * u1;
            FN(tsoftmax)(vd, 2, c->T, wd);
            REAL l0 = (j > 1) ? da[AIX(c, 0, i, j - 1)] : 0;
            REAL l2 = (j > 1) ? da[AIX(c, 2, i, j - 1)] : 0;
            da[AIX(c, 2, i, j)] = wd[0] * l0 + wd[1] * l2;
        }
    }
    FN(ksum_t) dk = {0, 0};
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st) {
                REAL lp = (c->a[AIX(c, st, i, j)] - S) / c->T;
                if (lp > 0) lp = 0;
                FN(kadd)(&dk, FN(clip_exp)(lp) * da[AIX(c, st, i, j)]);
            }
    REAL dS = dk.s;
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st) {
                size_t o = AIX(c, st, i, j);
                REAL lp = (c->a[o] - S) / c->T;
                if (lp > 0) lp = 0;
                be[o] = FN(clip_exp)(lp);
            }
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st) {
                size_t o = AIX(c, st, i, j);
                dbe[o] = be[o] * (da[o] - dS) / c->T;
            }
    for (int k = c->L1 + c->L2; k >= 2; --k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            REAL v = VV(i, j);
            int dg = (i > 1 && j > 1);
            FN(aff_cands)(c, c->a, i, j, vm, vi, vd);
            /* M */
            REAL bm = be[AIX(c, 0, i, j)], dbm = dbe[AIX(c, 0, i, j)];
            FN(tsoftmax)(vm, 4, c->T, wm);
            REAL tm[4];
            tm[0] = dg ? da[AIX(c, 0, i - 1, j - 1)] + v : 0;
            tm[1] = dg ? da[AIX(c, 1, i - 1, j - 1)] + v : 0;
            tm[2] = dg ? da[AIX(c, 2, i - 1, j - 1)] + v : 0;
            tm[3] = v;
            REAL swm = wm[0] * tm[0] + wm[1] * tm[1] + wm[2] * tm[2] + wm[3] * tm[3];
            REAL dwm[4];
            for (int q = 0; q < 4; ++q) dwm[q] = wm[q] * (tm[q] - swm) / c->T;
            H[(size_t)(i - 1) * c->ld + (j - 1)] += dbm * (wm[0] + wm[1] + wm[2] + wm[3]) +
                                                   bm * (dwm[0] + dwm[1] + dwm[2] + dwm[3]);
            if (dg) {
                for (int st = 0; st < 3; ++st) be[AIX(c, st, i - 1, j - 1)] += bm * wm[st];
                for (int st = 0; st < 3; ++st)
                    dbe[AIX(c, st, i - 1, j - 1)] += dbm * wm[st] + bm * dwm[st];
            }
            /* I */
            REAL bi = be[AIX(c, 1, i, j)], dbi = dbe[AIX(c, 1, i, j)];
            FN(tsoftmax)(vi, 2, c->T, wi);
            REAL ui[2];
            ui[0] = (i > 1) ? da[AIX(c, 0, i - 1, j)] : 0;
            ui[1] = (i > 1) ? da[AIX(c, 1, i - 1, j)] : 0;
            REAL swi = wi[0] * ui[0] + wi[1] * ui[1];
            REAL dwi0 = wi[0] * (ui[0] - swi) / c->T, dwi1 = wi[1] * (ui[1] - swi) / c->T;
            if (i > 1) {
                be[AIX(c, 0, i - 1, j)] += bi * wi[0];
                be[AIX(c, 1, i - 1, j)] += bi * wi[1];
                dbe[AIX(c, 0, i - 1, j)] += dbi * wi[0] + bi * dwi0;
                dbe[AIX(c, 1, i - 1, j)] += dbi * wi[1] + bi * dwi1;
            }
            /* D */
            REAL bd = be[AIX(c, 2, i, j)], dbd = dbe[AIX(c, 2, i, j)];
            FN(tsoftmax)(vd, 2, c->T, wd);
            REAL ud[2];
            ud[0] = (j > 1) ? da[AIX(c, 0, i, j - 1)] : 0;
            ud[1] = (j > 1) ? da[AIX(c, 2, i, j - 1)] : 0;
            REAL swd = wd[0] * ud[0] + wd[1] * ud[1];
            REAL dwd0 = wd[0] * (ud[0] - swd) / c->T, dwd1 = wd[1] * (ud[1] - swd) / c->T;
            if (j > 1) {
                be[AIX(c, 0, i, j - 1)] += bd * wd[0];
                be[AIX(c, 2, i, j - 1)] += bd * wd[1];
                dbe[AIX(c, 0, i, j - 1)] += dbd * wd[0] + bd * dwd0;
                dbe[AIX(c, 2, i, j - 1)] += dbd * wd[1] + bd * dwd1;
            }
        }
    }
#undef VV
}

/* d(post)/d(theta), theta in {gap_open, gap_ext, T}
 * (src/sw_affine/kernels_cpu.cpp:637-921): U = d(alpha)/d(theta) forward,
 * then beta and W = d(beta)/d(theta) backward; dP/dtheta += W_M. */
static void FN(aff_param)(const FN(aff_t) *c, REAL S, REAL dSdt, int pt, REAL *u,
                          REAL *be, REAL *w, REAL *dP, int L1max) {
    size_t n = 3 * c->plane;
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < n; ++q) { u[q] = 0; be[q] = 0; w[q] = 0; }
    for (size_t q = 0; q < nsc; ++q) dP[q] = 0;
    const REAL T = c->T;
    REAL vm[4], vi[2], vd[2], wm[4], wi[2], wd[2];
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            int dg = (i > 1 && j > 1);
            FN(aff_cands)(c, c->a, i, j, vm, vi, vd);
            FN(tsoftmax)(vm, 4, T, wm);
            REAL a0 = dg ? u[AIX(c, 0, i - 1, j - 1)] : 0;
            REAL a1 = dg ? u[AIX(c, 1, i - 1, j - 1)] : 0;
            REAL a2 = dg ? u[AIX(c, 2, i - 1, j - 1)] : 0;
            REAL um = wm[0] * a0 + wm[1] * a1 + wm[2] * a2;
            if (pt == 2) {
                REAL e = wm[0] * vm[0] + wm[1] * vm[1] + wm[2] * vm[2] + wm[3] * vm[3];
                um += (c->a[AIX(c, 0, i, j)] - e) / T;
            }
            u[AIX(c, 0, i, j)] = um;
            FN(tsoftmax)(vi, 2, T, wi);
            REAL b0 = (i > 1) ? u[AIX(c, 0, i - 1, j)] : 0;
            REAL b1 = (i > 1) ? u[AIX(c, 1, i - 1, j)] : 0;
            if (pt == 0) b0 += 1;
            if (pt == 1) b1 += 1;
            REAL ui = wi[0] * b0 + wi[1] * b1;
            if (pt == 2) {
                REAL e = wi[0] * vi[0] + wi[1] * vi[1];
                ui += (c->a[AIX(c, 1, i, j)] - e) / T;
            }
            u[AIX(c, 1, i, j)] = ui;
            FN(tsoftmax)(vd, 2, T, wd);
            REAL c0 = (j > 1) ? u[AIX(c, 0, i, j - 1)] : 0;
            REAL c2 = (j > 1) ? u[AIX(c, 2, i, j - 1)] : 0;
            if (pt == 0) c0 += 1;
            if (pt == 1) c2 += 1;
            REAL ud = wd[0] * c0 + wd[1] * c2;
            if (pt == 2) {
                REAL e = wd[0] * vd[0] + wd[1] * vd[1];
                ud += (c->a[AIX(c, 2, i, j)] - e) / T;
            }
            u[AIX(c, 2, i, j)] = ud;
        }
    }
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            for (int st = 0; st < 3; ++st)
                be[AIX(c, st, i, j)] = FN(end_weight)(c->a[AIX(c, st, i, j)], S, T);
    for (int k = c->L1 + c->L2; k >= 2; --k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            int dg = (i > 1 && j > 1);
            size_t om = AIX(c, 0, i, j), oi = AIX(c, 1, i, j), od = AIX(c, 2, i, j);
            FN(aff_cands)(c, c->a, i, j, vm, vi, vd);
            /* M */
            REAL bm = be[om];
            REAL bim = FN(end_weight)(c->a[om], S, T);
            REAL Wm = w[om] + bim * (u[om] - dSdt) / T;
            if (pt == 2 && c->a[om] > (REAL)NEG_BIG) Wm -= bim * (c->a[om] - S) / (T * T);
            FN(tsoftmax)(vm, 4, T, wm);
            REAL du[4];
            du[0] = dg ? u[AIX(c, 0, i - 1, j - 1)] : 0;
            du[1] = dg ? u[AIX(c, 1, i - 1, j - 1)] : 0;
            du[2] = dg ? u[AIX(c, 2, i - 1, j - 1)] : 0;
            du[3] = 0;
            REAL sw = wm[0] * du[0] + wm[1] * du[1] + wm[2] * du[2] + wm[3] * du[3];
            REAL dw[4];
            for (int q = 0; q < 4; ++q) dw[q] = wm[q] * (du[q] - sw) / T;
            if (pt == 2) {
                REAL e = wm[0] * vm[0] + wm[1] * vm[1] + wm[2] * vm[2] + wm[3] * vm[3];
                REAL it2 = (REAL)1 / (T * T);
                for (int q = 0; q < 4; ++q) dw[q] += wm[q] * (e - vm[q]) * it2;
            }
            dP[(size_t)(i - 1) * c->ld + (j - 1)] += Wm;
            if (dg) {
                for (int st = 0; st < 3; ++st) be[AIX(c, st, i - 1, j - 1)] += bm * wm[st];
                for (int st = 0; st < 3; ++st)
                    w[AIX(c, st, i - 1, j - 1)] += Wm * wm[st] + bm * dw[st];
            }
            /* I */
            REAL bi = be[oi];
            REAL bii = FN(end_weight)(c->a[oi], S, T);
            REAL Wi = w[oi] + bii * (u[oi] - dSdt) / T;
            if (pt == 2 && c->a[oi] > (REAL)NEG_BIG) Wi -= bii * (c->a[oi] - S) / (T * T);
            if (i > 1) {
                FN(tsoftmax)(vi, 2, T, wi);
                REAL e0 = u[AIX(c, 0, i - 1, j)], e1 = u[AIX(c, 1, i - 1, j)];
                if (pt == 0) e0 += 1;
                if (pt == 1) e1 += 1;
                REAL sI = wi[0] * e0 + wi[1] * e1;
                REAL d0 = wi[0] * (e0 - sI) / T, d1 = wi[1] * (e1 - sI) / T;
                if (pt == 2) {
                    REAL e = wi[0] * vi[0] + wi[1] * vi[1];
                    REAL it2 = (REAL)1 / (T * T);
                    d0 += wi[0] * (e - vi[0]) * it2;
                    d1 += wi[1] * (e - vi[1]) * it2;
                }
                be[AIX(c, 0, i - 1, j)] += bi * wi[0];
                be[AIX(c, 1, i - 1, j)] += bi * wi[1];
                w[AIX(c, 0, i - 1, j)] += Wi * wi[0] + bi * d0;
                w[AIX(c, 1, i - 1, j)] += Wi * wi[1] + bi * d1;
            }
            /* D */
            REAL bd = be[od];
            REAL bid = FN(end_weight)(c->a[od], S, T);
            REAL Wd = w[od] + bid * (u[od] - dSdt) / T;
            if (pt == 2 && c->a[od] > (REAL)NEG_BIG) Wd -= bid * (c->a[od] - S) / (T * T);
            if (j > 1) {
                FN(tsoftmax)(vd, 2, T, wd);
                REAL e0 = u[AIX(c, 0, i, j - 1)], e2 = u[AIX(c, 2, i, j - 1)];
                if (pt == 0) e0 += 1;
                if (pt == 1) e2 += 1;
                REAL sD = wd[0] * e0 + wd[1] * e2;
                REAL d0 = wd[0] * (e0 - sD) / T, d2 = wd[1] * (e2 - sD) / T;
                if (pt == 2) {
                    REAL e = wd[0] * vd[0] + wd[1] * vd[1];
                    REAL it2 = (REAL)1 / (T * T);
                    d0 += wd[0] * (e - vd[0]) * it2;
                    d2 += wd[1] * (e - vd[1]) * it2;
                }
                be[AIX(c, 0, i, j - 1)] += bd * wd[0];
                be[AIX(c, 2, i, j - 1)] += bd * wd[1];
                w[AIX(c, 0, i, j - 1)] += Wd * wd[0] + bd * d0;
                w[AIX(c, 2, i, j - 1)] += Wd * wd[1] + bd * d2;
            }
        }
    }
}

/* ---- linear model ------------------------------------------------------ */

#define LIX(c, i, j) ((size_t)(i) * (c)->cols + (size_t)(j))

typedef struct {
    int L1, L2, ld;
    const REAL *s;
    REAL g, T;
    size_t cols;
    REAL *a;
} FN(lin_t);

/* align, up, left, sky candidates of cell (i,j) (src/sw/kernels_cpu.cpp:112-121). */
static void FN(lin_cands)(const FN(lin_t) *c, const REAL *tab, int i, int j, REAL v[4]) {
    REAL s = SC(c, i, j);
    v[0] = (i > 1 && j > 1) ? tab[LIX(c, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    v[1] = (i > 1) ? tab[LIX(c, i - 1, j)] + c->g : (REAL)NEG_BIG;
    v[2] = (j > 1) ? tab[LIX(c, i, j - 1)] + c->g : (REAL)NEG_BIG;
    v[3] = s;
}

/* src/sw/kernels_cpu.cpp:70-148 */
static REAL FN(lin_forward)(FN(lin_t) *c) {
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    for (size_t q = 0; q < n; ++q) c->a[q] = (REAL)NEG_BIG;
    c->a[0] = 0;
    REAL v[4];
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            FN(lin_cands)(c, c->a, i, j, v);
            c->a[LIX(c, i, j)] = FN(tlse)(v, 4, c->T);
        }
    REAL m = (REAL)NEG_BIG;
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j)
            if (c->a[LIX(c, i, j)] > m) m = c->a[LIX(c, i, j)];
    FN(ksum_t) k = {0, 0};
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j) {
            REAL x = c->a[LIX(c, i, j)];
            if (x > (REAL)NEG_BIG) FN(kadd)(&k, FN(clip_exp)((x - m) / c->T));
        }
    return m + c->T * LOGF(k.s);
}

/* src/sw/kernels_cpu.cpp:154-271; g[0]=dS/dgap, g[1]=dS/dT. */
static void FN(lin_adjoint)(const FN(lin_t) *c, REAL S, REAL *be, REAL *post, int L1max,
                            REAL g[2]) {
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < nsc; ++q) post[q] = 0;
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j) {
            REAL lp = (c->a[LIX(c, i, j)] - S) / c->T;
            if (lp > 0) lp = 0;
            be[LIX(c, i, j)] = FN(clip_exp)(lp);
        }
    REAL ggap = 0;
    REAL v[4], w[4];
    for (int k = c->L1 + c->L2; k >= 2; --k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            REAL b = be[LIX(c, i, j)];
            if (!FN(live)(b)) continue;
            FN(lin_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 4, c->T, w);
            post[(size_t)(i - 1) * c->ld + (j - 1)] += b * (w[0] + w[3]);
            if (i > 1 && j > 1 && w[0] > 0) be[LIX(c, i - 1, j - 1)] += b * w[0];
            if (i > 1 && w[1] > 0) { be[LIX(c, i - 1, j)] += b * w[1]; ggap += b * w[1]; }
            if (j > 1 && w[2] > 0) { be[LIX(c, i, j - 1)] += b * w[2]; ggap += b * w[2]; }
        }
    }
    FN(ksum_t) ms = {0, 0};
    for (size_t q = 0; q < nsc; ++q) FN(kadd)(&ms, post[q] * c->s[q]);
    REAL total = ms.s + ggap * c->g;
    g[0] = ggap;
    g[1] = (S - total) / c->T;
}

/* Softmax of the four linear candidates with a plain (uncompensated) sum and
 * a 1e-20 guard, as the linear parameter-Jacobian uses
 * (src/sw/kernels_cpu.cpp:547-560).  Returns 0 when every candidate is dead. */
static int FN(lin_plain_softmax)(const REAL v[4], REAL T, REAL w[4]) {
    REAL m = FN(vmax)(v, 4);
    if (m <= (REAL)NEG_BIG) return 0;
    for (int q = 0; q < 4; ++q) w[q] = FN(clip_exp)((v[q] - m) / T);
    REAL sum = w[0] + w[1] + w[2] + w[3];
    REAL inv = (sum > (REAL)1e-20) ? (REAL)1 / sum : (REAL)0;
    for (int q = 0; q < 4; ++q) w[q] *= inv;
    return 1;
}

/* src/sw/kernels_cpu.cpp:279-485 (HVP of the linear model). */
static void FN(lin_hvp)(const FN(lin_t) *c, REAL S, const REAL *V, REAL *da, REAL *be,
                        REAL *dbe, REAL *H, int L1max) {
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < n; ++q) { da[q] = 0; be[q] = 0; dbe[q] = 0; }
    for (size_t q = 0; q < nsc; ++q) H[q] = 0;
    REAL v[4], w[4];
#define VV(i, j) V[(size_t)((i) - 1) * c->ld + (size_t)((j) - 1)]
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            REAL vv = VV(i, j);
            FN(lin_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 4, c->T, w);
            REAL t0 = (i > 1 && j > 1) ? da[LIX(c, i - 1, j - 1)] + vv : 0;
            REAL t1 = (i > 1) ? da[LIX(c, i - 1, j)] : 0;
            REAL t2 = (j > 1) ? da[LIX(c, i, j - 1)] : 0;
            da[LIX(c, i, j)] = w[0] * t0 + w[1] * t1 + w[2] * t2 + w[3] * vv;
        }
    }
    FN(ksum_t) dk = {0, 0};
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j) {
            REAL lp = (c->a[LIX(c, i, j)] - S) / c->T;
            if (lp > 0) lp = 0;
            FN(kadd)(&dk, FN(clip_exp)(lp) * da[LIX(c, i, j)]);
        }
    REAL dS = dk.s;
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j) {
            size_t o = LIX(c, i, j);
            REAL lp = (c->a[o] - S) / c->T;
            if (lp > 0) lp = 0;
            be[o] = FN(clip_exp)(lp);
        }
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j) {
            size_t o = LIX(c, i, j);
            dbe[o] = be[o] * (da[o] - dS) / c->T;
        }
    for (int k = c->L1 + c->L2; k >= 2; --k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            REAL vv = VV(i, j);
            size_t o = LIX(c, i, j);
            REAL b = be[o], db = dbe[o];
            if (!FN(live)(b)) continue;
            FN(lin_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 4, c->T, w);
            REAL t[4];
            t[0] = (i > 1 && j > 1) ? da[LIX(c, i - 1, j - 1)] + vv : 0;
            t[1] = (i > 1) ? da[LIX(c, i - 1, j)] : 0;
            t[2] = (j > 1) ? da[LIX(c, i, j - 1)] : 0;
            t[3] = vv;
            REAL sw = w[0] * t[0] + w[1] * t[1] + w[2] * t[2] + w[3] * t[3];
            REAL dw[4];
            for (int q = 0; q < 4; ++q) dw[q] = w[q] * (t[q] - sw) / c->T;
            H[(size_t)(i - 1) * c->ld + (j - 1)] += db * (w[0] + w[3]) + b * (dw[0] + dw[3]);
            if (i > 1 && j > 1 && w[0] > 0) be[LIX(c, i - 1, j - 1)] += b * w[0];
            if (i > 1 && w[1] > 0) be[LIX(c, i - 1, j)] += b * w[1];
            if (j > 1 && w[2] > 0) be[LIX(c, i, j - 1)] += b * w[2];
            if (i > 1 && j > 1 && w[0] > 0) dbe[LIX(c, i - 1, j - 1)] += db * w[0] + b * dw[0];
            if (i > 1 && w[1] > 0) dbe[LIX(c, i - 1, j)] += db * w[1] + b * dw[1];
            if (j > 1 && w[2] > 0) dbe[LIX(c, i, j - 1)] += db * w[2] + b * dw[2];
        }
    }
#undef VV
}

/* src/sw/kernels_cpu.cpp:491-710 (dP/dtheta, theta in {gap, T}). */
static void FN(lin_param)(const FN(lin_t) *c, REAL S, REAL dSdt, int pt, REAL *u, REAL *be,
                          REAL *wt, REAL *dP, int L1max) {
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < n; ++q) { u[q] = 0; be[q] = 0; wt[q] = 0; }
    for (size_t q = 0; q < nsc; ++q) dP[q] = 0;
    const REAL T = c->T;
    REAL v[4], w[4];
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            FN(lin_cands)(c, c->a, i, j, v);
            if (!FN(lin_plain_softmax)(v, T, w)) { u[LIX(c, i, j)] = 0; continue; }
            REAL a0 = (i > 1 && j > 1) ? u[LIX(c, i - 1, j - 1)] : 0;
            REAL a1 = (i > 1) ? u[LIX(c, i - 1, j)] : 0;
            REAL a2 = (j > 1) ? u[LIX(c, i, j - 1)] : 0;
            if (pt == 0) { a1 += 1; a2 += 1; }
            REAL du = w[0] * a0 + w[1] * a1 + w[2] * a2 + w[3] * 0;
            if (pt == 1) {
                REAL e = w[0] * v[0] + w[1] * v[1] + w[2] * v[2] + w[3] * v[3];
                du += (c->a[LIX(c, i, j)] - e) / T;
            }
            u[LIX(c, i, j)] = du;
        }
    }
    for (int i = 0; i <= c->L1; ++i)
        for (int j = 0; j <= c->L2; ++j) {
            REAL lp = (c->a[LIX(c, i, j)] - S) / T;
            if (lp > 0) lp = 0;
            be[LIX(c, i, j)] = FN(clip_exp)(lp);
        }
    for (int k = c->L1 + c->L2; k >= 2; --k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            if (j < 1 || j > c->L2) continue;
            size_t o = LIX(c, i, j);
            REAL b = be[o];
            REAL b0 = 0;
            if (c->a[o] > (REAL)NEG_BIG) {
                REAL lp = (c->a[o] - S) / T;
                if (lp > 0) lp = 0;
                b0 = FN(clip_exp)(lp);
            }
            REAL dW = b0 * (u[o] - dSdt) / T;
            if (pt == 1 && c->a[o] > (REAL)NEG_BIG) dW -= b0 * (c->a[o] - S) / (T * T);
            REAL W = wt[o] + dW;
            if (b <= (REAL)1e-20 && FABS(W) <= (REAL)1e-20) continue;
            FN(lin_cands)(c, c->a, i, j, v);
            if (!FN(lin_plain_softmax)(v, T, w)) continue;
            REAL du[4];
            du[0] = (i > 1 && j > 1) ? u[LIX(c, i - 1, j - 1)] : 0;
            du[1] = (i > 1) ? u[LIX(c, i - 1, j)] : 0;
            du[2] = (j > 1) ? u[LIX(c, i, j - 1)] : 0;
            du[3] = 0;
            if (pt == 0) { du[1] += 1; du[2] += 1; }
            REAL sw = w[0] * du[0] + w[1] * du[1] + w[2] * du[2] + w[3] * du[3];
            REAL dw[4];
            for (int q = 0; q < 4; ++q) dw[q] = w[q] * (du[q] - sw) / T;
            if (pt == 1) {
                REAL e = w[0] * v[0] + w[1] * v[1] + w[2] * v[2] + w[3] * v[3];
                REAL it2 = (REAL)1 / (T * T);
                for (int q = 0; q < 4; ++q) dw[q] += w[q] * (e - v[q]) * it2;
            }
            dP[(size_t)(i - 1) * c->ld + (j - 1)] += W * (w[0] + w[3]) + b * (dw[0] + dw[3]);
            if (v[0] > (REAL)NEG_BIG) {
                be[LIX(c, i - 1, j - 1)] += b * w[0];
                wt[LIX(c, i - 1, j - 1)] += W * w[0] + b * dw[0];
            }
            if (v[1] > (REAL)NEG_BIG) {
                be[LIX(c, i - 1, j)] += b * w[1];
                wt[LIX(c, i - 1, j)] += W * w[1] + b * dw[1];
            }
            if (v[2] > (REAL)NEG_BIG) {
                be[LIX(c, i, j - 1)] += b * w[2];
                wt[LIX(c, i, j - 1)] += W * w[2] + b * dw[2];
            }
        }
    }
}

/* ---- global alignment (Needleman-Wunsch), linear gap -------------------
 * Same table layout as the linear model (lin_t).  Boundaries A[0,0] = 0,
 * A[i,0] = i*gap, A[0,j] = j*gap; three candidates (diag + s, up + gap,
 * left + gap), no local start; S = A[L1, L2]; beta = 1 at the terminal only.
 * Loop orders follow src/nw/kernels_cpu.cpp so that the float instantiation
 * accumulates in the same order as the reference. */

static void FN(nw_cands)(const FN(lin_t) *c, const REAL *tab, int i, int j, REAL v[3]) {
    v[0] = tab[LIX(c, i - 1, j - 1)] + SC(c, i, j);
    v[1] = tab[LIX(c, i - 1, j)] + c->g;
    v[2] = tab[LIX(c, i, j - 1)] + c->g;
}

static void FN(nw_bounds)(FN(lin_t) *c, REAL *tab, int gap_index) {
    /* gap_index: boundary values i*gap (0) or d/dgap of them, i (1) */
    tab[0] = 0;
    for (int i = 1; i <= c->L1; ++i) tab[LIX(c, i, 0)] = gap_index ? (REAL)i : (REAL)i * c->g;
    for (int j = 1; j <= c->L2; ++j) tab[LIX(c, 0, j)] = gap_index ? (REAL)j : (REAL)j * c->g;
}

/* src/nw/kernels_cpu.cpp:77-150 */
static REAL FN(nw_forward)(FN(lin_t) *c) {
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    for (size_t q = 0; q < n; ++q) c->a[q] = (REAL)NEG_BIG;
    FN(nw_bounds)(c, c->a, 0);
    REAL v[3];
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            FN(nw_cands)(c, c->a, i, j, v);
            c->a[LIX(c, i, j)] = FN(tlse)(v, 3, c->T);
        }
    return c->a[LIX(c, c->L1, c->L2)];
}

#define NW_DIAGS(c, k, i, j)                                                  \
    for (int k = (c)->L1 + (c)->L2; k >= 2; --k)                              \
        for (int i = ((k - (c)->L2 > 1) ? k - (c)->L2 : 1),                   \
                 i##_end = (((c)->L1 < k - 1) ? (c)->L1 : k - 1);             \
             i <= i##_end; ++i)                                               \
            for (int j = k - i, j##_once = 1; j##_once; j##_once = 0)

/* src/nw/kernels_cpu.cpp:156-268; g[0] = dS/dgap, g[1] = dS/dT. */
static void FN(nw_adjoint)(const FN(lin_t) *c, REAL S, REAL *be, REAL *post, int L1max,
                           REAL g[2]) {
    size_t nsc = (size_t)L1max * c->ld;
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    for (size_t q = 0; q < nsc; ++q) post[q] = 0;
    for (size_t q = 0; q < n; ++q) be[q] = 0;
    be[LIX(c, c->L1, c->L2)] = 1;
    FN(ksum_t) gs = {0, 0}, ms = {0, 0};
    REAL v[3], w[3];
    NW_DIAGS(c, k, i, j) {
        REAL b = be[LIX(c, i, j)];
        if (b == 0) continue;
        REAL sc = SC(c, i, j);
        FN(nw_cands)(c, c->a, i, j, v);
        FN(tsoftmax)(v, 3, c->T, w);
        REAL p = b * w[0];
        post[(size_t)(i - 1) * c->ld + (j - 1)] = p;
        FN(kadd)(&ms, p * sc);
        FN(kadd)(&gs, b * (w[1] + w[2]));
        if (w[0] > 0) be[LIX(c, i - 1, j - 1)] += b * w[0];
        if (w[1] > 0) be[LIX(c, i - 1, j)] += b * w[1];
        if (w[2] > 0) be[LIX(c, i, j - 1)] += b * w[2];
    }
    /* boundary cells carry gap costs i*gap and j*gap (kernels_cpu.cpp:250-258) */
    for (int i = 1; i <= c->L1; ++i) FN(kadd)(&gs, be[LIX(c, i, 0)] * (REAL)i);
    for (int j = 1; j <= c->L2; ++j) FN(kadd)(&gs, be[LIX(c, 0, j)] * (REAL)j);
    REAL gg = gs.s;
    g[0] = gg;
    g[1] = (S - (ms.s + gg * c->g)) / c->T;
}

/* src/nw/kernels_cpu.cpp:276-437 (HVP). */
static void FN(nw_hvp)(const FN(lin_t) *c, const REAL *V, REAL *da, REAL *be, REAL *dbe,
                       REAL *H, int L1max) {
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < n; ++q) { da[q] = 0; be[q] = 0; dbe[q] = 0; }
    for (size_t q = 0; q < nsc; ++q) H[q] = 0;
    REAL v[3], w[3];
#define VV(i, j) V[(size_t)((i) - 1) * c->ld + (size_t)((j) - 1)]
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            FN(nw_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 3, c->T, w);
            REAL d0 = da[LIX(c, i - 1, j - 1)] + VV(i, j);
            REAL d1 = da[LIX(c, i - 1, j)];
            REAL d2 = da[LIX(c, i, j - 1)];
            da[LIX(c, i, j)] = w[0] * d0 + w[1] * d1 + w[2] * d2;
        }
    be[LIX(c, c->L1, c->L2)] = 1;
    NW_DIAGS(c, k, i, j) {
        size_t o = LIX(c, i, j);
        REAL b = be[o], db = dbe[o];
        if (b == 0 && FABS(db) < (REAL)1e-20) continue;
        FN(nw_cands)(c, c->a, i, j, v);
        FN(tsoftmax)(v, 3, c->T, w);
        REAL t[3];
        t[0] = da[LIX(c, i - 1, j - 1)] + VV(i, j);
        t[1] = da[LIX(c, i - 1, j)];
        t[2] = da[LIX(c, i, j - 1)];
        REAL e = w[0] * t[0] + w[1] * t[1] + w[2] * t[2];
        REAL dw[3];
        for (int q = 0; q < 3; ++q) dw[q] = w[q] * (t[q] - e) / c->T;
        H[(size_t)(i - 1) * c->ld + (j - 1)] = db * w[0] + b * dw[0];
        if (w[0] > 0) { be[LIX(c, i - 1, j - 1)] += b * w[0]; dbe[LIX(c, i - 1, j - 1)] += db * w[0] + b * dw[0]; }
        if (w[1] > 0) { be[LIX(c, i - 1, j)] += b * w[1]; dbe[LIX(c, i - 1, j)] += db * w[1] + b * dw[1]; }
        if (w[2] > 0) { be[LIX(c, i, j - 1)] += b * w[2]; dbe[LIX(c, i, j - 1)] += db * w[2] + b * dw[2]; }
    }
#undef VV
}

/* src/nw/kernels_cpu.cpp:445-640 (dP/dtheta, theta in {gap, T}). */
static void FN(nw_param)(FN(lin_t) *c, int pt, REAL *u, REAL *be, REAL *wt, REAL *dP,
                         int L1max) {
    size_t n = (size_t)(c->L1 + 1) * c->cols;
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < n; ++q) { u[q] = 0; be[q] = 0; wt[q] = 0; }
    for (size_t q = 0; q < nsc; ++q) dP[q] = 0;
    if (pt == 0) FN(nw_bounds)(c, u, 1);
    const REAL T = c->T;
    REAL v[3], w[3];
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            FN(nw_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 3, T, w);
            REAL a0 = u[LIX(c, i - 1, j - 1)], a1 = u[LIX(c, i - 1, j)], a2 = u[LIX(c, i, j - 1)];
            if (pt == 0) { a1 += 1; a2 += 1; }
            REAL U = w[0] * a0 + w[1] * a1 + w[2] * a2;
            if (pt == 1) {
                REAL e = w[0] * v[0] + w[1] * v[1] + w[2] * v[2];
                U += (c->a[LIX(c, i, j)] - e) / T;
            }
            u[LIX(c, i, j)] = U;
        }
    be[LIX(c, c->L1, c->L2)] = 1;
    NW_DIAGS(c, k, i, j) {
        size_t o = LIX(c, i, j);
        REAL b = be[o], W = wt[o];
        if (b == 0 && FABS(W) < (REAL)1e-20) continue;
        FN(nw_cands)(c, c->a, i, j, v);
        FN(tsoftmax)(v, 3, T, w);
        REAL du[3] = {u[LIX(c, i - 1, j - 1)], u[LIX(c, i - 1, j)], u[LIX(c, i, j - 1)]};
        if (pt == 0) { du[1] += 1; du[2] += 1; }
        REAL e = w[0] * du[0] + w[1] * du[1] + w[2] * du[2];
        REAL dw[3];
        for (int q = 0; q < 3; ++q) dw[q] = w[q] * (du[q] - e) / T;
        if (pt == 1) {
            REAL ev = w[0] * v[0] + w[1] * v[1] + w[2] * v[2];
            REAL it2 = (REAL)1 / (T * T);
            for (int q = 0; q < 3; ++q) dw[q] += w[q] * (ev - v[q]) * it2;
        }
        dP[(size_t)(i - 1) * c->ld + (j - 1)] = W * w[0] + b * dw[0];
        if (w[0] > 0) { be[LIX(c, i - 1, j - 1)] += b * w[0]; wt[LIX(c, i - 1, j - 1)] += W * w[0] + b * dw[0]; }
        if (w[1] > 0) { be[LIX(c, i - 1, j)] += b * w[1]; wt[LIX(c, i - 1, j)] += W * w[1] + b * dw[1]; }
        if (w[2] > 0) { be[LIX(c, i, j - 1)] += b * w[2]; wt[LIX(c, i, j - 1)] += W * w[2] + b * dw[2]; }
    }
}

/* ---- global alignment, affine gaps (Needleman-Wunsch affine) ------------
 * Three states on the affine tables (aff_t): M = s + LSE(M, I, D at diag),
 * I = LSE(M + go, I + ge, D + go) from above, D = LSE(M + go, I + go, D + ge)
 * from the left.  Boundaries M(0,0) = 0, I(i,0) = go + (i-1) ge,
 * D(0,j) = go + (j-1) ge, every other boundary state NEG_BIG.  S = LSE of the
 * three states at (L1, L2).  The helpers are the file's own
 * (src/nw_affine/kernels_cpu.cpp:37-98): the LSE skips NEG_BIG terms in its
 * Kahan sum, the weights use a plain sum. */

static REAL FN(nwa_lse3)(REAL a, REAL b, REAL c, REAL T) {
    REAL m = a > b ? a : b;
    if (c > m) m = c;
    if (m <= (REAL)NEG_BIG) return (REAL)NEG_BIG;
    FN(ksum_t) k = {0, 0};
    if (a > (REAL)NEG_BIG) FN(kadd)(&k, FN(clip_exp)((a - m) / T));
    if (b > (REAL)NEG_BIG) FN(kadd)(&k, FN(clip_exp)((b - m) / T));
    if (c > (REAL)NEG_BIG) FN(kadd)(&k, FN(clip_exp)((c - m) / T));
    if (k.s <= 0) return (REAL)NEG_BIG;
    return m + T * LOGF(k.s);
}

static void FN(nwa_w3)(REAL a, REAL b, REAL c, REAL T, REAL w[3]) {
    REAL m = a > b ? a : b;
    if (c > m) m = c;
    w[0] = w[1] = w[2] = 0;
    if (m <= (REAL)NEG_BIG) return;
    REAL ea = a > (REAL)NEG_BIG ? FN(clip_exp)((a - m) / T) : 0;
    REAL eb = b > (REAL)NEG_BIG ? FN(clip_exp)((b - m) / T) : 0;
    REAL ec = c > (REAL)NEG_BIG ? FN(clip_exp)((c - m) / T) : 0;
    REAL t = ea + eb + ec;
    if (t > 0) { w[0] = ea / t; w[1] = eb / t; w[2] = ec / t; }
}

/* candidates of cell (i,j): v[0..2] diag M, I, D; v[3..5] up M+go, I+ge, D+go;
 * v[6..8] left M+go, I+go, D+ge */
static void FN(nwa_cands)(const FN(aff_t) *c, const REAL *t, int i, int j, REAL v[9]) {
    v[0] = t[AIX(c, 0, i - 1, j - 1)]; v[1] = t[AIX(c, 1, i - 1, j - 1)]; v[2] = t[AIX(c, 2, i - 1, j - 1)];
    v[3] = t[AIX(c, 0, i - 1, j)] + c->go; v[4] = t[AIX(c, 1, i - 1, j)] + c->ge;
    v[5] = t[AIX(c, 2, i - 1, j)] + c->go;
    v[6] = t[AIX(c, 0, i, j - 1)] + c->go; v[7] = t[AIX(c, 1, i, j - 1)] + c->go;
    v[8] = t[AIX(c, 2, i, j - 1)] + c->ge;
}

/* src/nw_affine/kernels_cpu.cpp:100-187 */
static REAL FN(nwa_forward)(FN(aff_t) *c) {
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) c->a[AIX(c, st, i, j)] = (REAL)NEG_BIG;
    c->a[AIX(c, 0, 0, 0)] = 0;
    for (int i = 1; i <= c->L1; ++i) c->a[AIX(c, 1, i, 0)] = c->go + (REAL)(i - 1) * c->ge;
    for (int j = 1; j <= c->L2; ++j) c->a[AIX(c, 2, 0, j)] = c->go + (REAL)(j - 1) * c->ge;
    REAL v[9];
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            FN(nwa_cands)(c, c->a, i, j, v);
            c->a[AIX(c, 0, i, j)] = SC(c, i, j) + FN(nwa_lse3)(v[0], v[1], v[2], c->T);
            c->a[AIX(c, 1, i, j)] = FN(nwa_lse3)(v[3], v[4], v[5], c->T);
            c->a[AIX(c, 2, i, j)] = FN(nwa_lse3)(v[6], v[7], v[8], c->T);
        }
    return FN(nwa_lse3)(c->a[AIX(c, 0, c->L1, c->L2)], c->a[AIX(c, 1, c->L1, c->L2)],
                        c->a[AIX(c, 2, c->L1, c->L2)], c->T);
}

#define NWA_TH ((REAL)1e-20)

/* src/nw_affine/kernels_cpu.cpp:193-347; g = dS/d(go, ge, T). */
static void FN(nwa_adjoint)(const FN(aff_t) *c, REAL S, REAL *be, REAL *post, int L1max,
                            REAL g[3]) {
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < nsc; ++q) post[q] = 0;
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) be[AIX(c, st, i, j)] = 0;
    const REAL T = c->T;
    REAL w[3], v[9];
    FN(nwa_w3)(c->a[AIX(c, 0, c->L1, c->L2)], c->a[AIX(c, 1, c->L1, c->L2)],
               c->a[AIX(c, 2, c->L1, c->L2)], T, w);
    for (int st = 0; st < 3; ++st) be[AIX(c, st, c->L1, c->L2)] = w[st];
    REAL so = 0, se = 0;
    FN(ksum_t) ms = {0, 0};
    NW_DIAGS(c, k, i, j) {
        REAL bM = be[AIX(c, 0, i, j)], bI = be[AIX(c, 1, i, j)], bD = be[AIX(c, 2, i, j)];
        REAL sc = SC(c, i, j);
        FN(nwa_cands)(c, c->a, i, j, v);
        if (bM > NWA_TH && FN(nwa_lse3)(v[0], v[1], v[2], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[0], v[1], v[2], T, w);
            for (int st = 0; st < 3; ++st)
                if (v[st] > (REAL)NEG_BIG) be[AIX(c, st, i - 1, j - 1)] += bM * w[st];
            post[(size_t)(i - 1) * c->ld + (j - 1)] += bM;
            FN(kadd)(&ms, bM * sc);
        }
        if (bI > NWA_TH && FN(nwa_lse3)(v[3], v[4], v[5], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[3], v[4], v[5], T, w);
            for (int st = 0; st < 3; ++st) be[AIX(c, st, i - 1, j)] += bI * w[st];
            so += bI * (w[0] + w[2]);
            se += bI * w[1];
        }
        if (bD > NWA_TH && FN(nwa_lse3)(v[6], v[7], v[8], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[6], v[7], v[8], T, w);
            for (int st = 0; st < 3; ++st) be[AIX(c, st, i, j - 1)] += bD * w[st];
            so += bD * (w[0] + w[1]);
            se += bD * w[2];
        }
    }
    /* leading-gap boundary states (kernels_cpu.cpp:318-335) */
    for (int i = 1; i <= c->L1; ++i) {
        REAL b = be[AIX(c, 1, i, 0)];
        if (b > NWA_TH) { so += b; se += b * (REAL)(i - 1); }
    }
    for (int j = 1; j <= c->L2; ++j) {
        REAL b = be[AIX(c, 2, 0, j)];
        if (b > NWA_TH) { so += b; se += b * (REAL)(j - 1); }
    }
    g[0] = so;
    g[1] = se;
    g[2] = (S - (ms.s + so * c->go + se * c->ge)) / T;
}

/* dw = w (t - sum w t) / T over three terms, left to right as the reference */
static void FN(nwa_dw)(const REAL w[3], const REAL t[3], REAL T, REAL dw[3]) {
    REAL e = w[0] * t[0] + w[1] * t[1] + w[2] * t[2];
    for (int q = 0; q < 3; ++q) dw[q] = w[q] * (t[q] - e) / T;
}

/* src/nw_affine/kernels_cpu.cpp:353-613 (HVP). */
static void FN(nwa_hvp)(FN(aff_t) *c, const REAL *V, REAL *da, REAL *be, REAL *dbe, REAL *H,
                        int L1max) {
    size_t nsc = (size_t)L1max * c->ld;
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) {
                size_t o = AIX(c, st, i, j);
                da[o] = 0; be[o] = 0; dbe[o] = 0;
            }
    for (size_t q = 0; q < nsc; ++q) H[q] = 0;
    const REAL T = c->T;
    REAL w[3], v[9], t[3], dw[3];
#define VV(i, j) V[(size_t)((i) - 1) * c->ld + (size_t)((j) - 1)]
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            FN(nwa_cands)(c, c->a, i, j, v);
            if (FN(nwa_lse3)(v[0], v[1], v[2], T) > (REAL)NEG_BIG) {
                FN(nwa_w3)(v[0], v[1], v[2], T, w);
                da[AIX(c, 0, i, j)] = VV(i, j) + w[0] * da[AIX(c, 0, i - 1, j - 1)] +
                                      w[1] * da[AIX(c, 1, i - 1, j - 1)] + w[2] * da[AIX(c, 2, i - 1, j - 1)];
            } else {
                da[AIX(c, 0, i, j)] = 0;
            }
            if (FN(nwa_lse3)(v[3], v[4], v[5], T) > (REAL)NEG_BIG) {
                FN(nwa_w3)(v[3], v[4], v[5], T, w);
                da[AIX(c, 1, i, j)] = w[0] * da[AIX(c, 0, i - 1, j)] + w[1] * da[AIX(c, 1, i - 1, j)] +
                                      w[2] * da[AIX(c, 2, i - 1, j)];
            } else {
                da[AIX(c, 1, i, j)] = 0;
            }
            if (FN(nwa_lse3)(v[6], v[7], v[8], T) > (REAL)NEG_BIG) {
                FN(nwa_w3)(v[6], v[7], v[8], T, w);
                da[AIX(c, 2, i, j)] = w[0] * da[AIX(c, 0, i, j - 1)] + w[1] * da[AIX(c, 1, i, j - 1)] +
                                      w[2] * da[AIX(c, 2, i, j - 1)];
            } else {
                da[AIX(c, 2, i, j)] = 0;
            }
        }
    }
    {
        size_t f0 = AIX(c, 0, c->L1, c->L2), f1 = AIX(c, 1, c->L1, c->L2), f2 = AIX(c, 2, c->L1, c->L2);
        FN(nwa_w3)(c->a[f0], c->a[f1], c->a[f2], T, w);
        be[f0] = w[0]; be[f1] = w[1]; be[f2] = w[2];
        t[0] = da[f0]; t[1] = da[f1]; t[2] = da[f2];
        FN(nwa_dw)(w, t, T, dw);
        dbe[f0] = dw[0]; dbe[f1] = dw[1]; dbe[f2] = dw[2];
    }
    NW_DIAGS(c, k, i, j) {
        REAL bM = be[AIX(c, 0, i, j)], bI = be[AIX(c, 1, i, j)], bD = be[AIX(c, 2, i, j)];
        REAL dM = dbe[AIX(c, 0, i, j)], dI = dbe[AIX(c, 1, i, j)], dD = dbe[AIX(c, 2, i, j)];
        FN(nwa_cands)(c, c->a, i, j, v);
        if ((bM > NWA_TH || FABS(dM) > NWA_TH) && FN(nwa_lse3)(v[0], v[1], v[2], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[0], v[1], v[2], T, w);
            for (int st = 0; st < 3; ++st) t[st] = da[AIX(c, st, i - 1, j - 1)];
            FN(nwa_dw)(w, t, T, dw);
            for (int st = 0; st < 3; ++st)
                if (v[st] > (REAL)NEG_BIG) {
                    be[AIX(c, st, i - 1, j - 1)] += bM * w[st];
                    dbe[AIX(c, st, i - 1, j - 1)] += dM * w[st] + bM * dw[st];
                }
            H[(size_t)(i - 1) * c->ld + (j - 1)] += dM;
        }
        if ((bI > NWA_TH || FABS(dI) > NWA_TH) && FN(nwa_lse3)(v[3], v[4], v[5], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[3], v[4], v[5], T, w);
            for (int st = 0; st < 3; ++st) t[st] = da[AIX(c, st, i - 1, j)];
            FN(nwa_dw)(w, t, T, dw);
            for (int st = 0; st < 3; ++st) {
                be[AIX(c, st, i - 1, j)] += bI * w[st];
                dbe[AIX(c, st, i - 1, j)] += dI * w[st] + bI * dw[st];
            }
        }
        if ((bD > NWA_TH || FABS(dD) > NWA_TH) && FN(nwa_lse3)(v[6], v[7], v[8], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[6], v[7], v[8], T, w);
            for (int st = 0; st < 3; ++st) t[st] = da[AIX(c, st, i, j - 1)];
            FN(nwa_dw)(w, t, T, dw);
            for (int st = 0; st < 3; ++st) {
                be[AIX(c, st, i, j - 1)] += bD * w[st];
                dbe[AIX(c, st, i, j - 1)] += dD * w[st] + bD * dw[st];
            }
        }
    }
#undef VV
}

/* src/nw_affine/kernels_cpu.cpp:619-1000 (dP/dtheta, theta in {go, ge, T}). */
static void FN(nwa_param)(FN(aff_t) *c, int pt, REAL *u, REAL *be, REAL *wt, REAL *dP,
                          int L1max) {
    size_t nsc = (size_t)L1max * c->ld;
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) {
                size_t o = AIX(c, st, i, j);
                u[o] = 0; be[o] = 0; wt[o] = 0;
            }
    for (size_t q = 0; q < nsc; ++q) dP[q] = 0;
    if (pt == 0 || pt == 1) {
        for (int i = 1; i <= c->L1; ++i) u[AIX(c, 1, i, 0)] = pt == 0 ? (REAL)1 : (REAL)(i - 1);
        for (int j = 1; j <= c->L2; ++j) u[AIX(c, 2, 0, j)] = pt == 0 ? (REAL)1 : (REAL)(j - 1);
    }
    const REAL T = c->T;
    /* direct tangents of the gap terms: I from (M, I, D) up, D from (M, I, D) left */
    const REAL dI[3] = {pt == 0 ? 1 : 0, pt == 1 ? 1 : 0, pt == 0 ? 1 : 0};
    const REAL dD[3] = {pt == 0 ? 1 : 0, pt == 0 ? 1 : 0, pt == 1 ? 1 : 0};
    REAL w[3], v[9], t[3], dw[3];
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            FN(nwa_cands)(c, c->a, i, j, v);
            if (FN(nwa_lse3)(v[0], v[1], v[2], T) > (REAL)NEG_BIG) {
                FN(nwa_w3)(v[0], v[1], v[2], T, w);
                REAL U = w[0] * u[AIX(c, 0, i - 1, j - 1)] + w[1] * u[AIX(c, 1, i - 1, j - 1)] +
                         w[2] * u[AIX(c, 2, i - 1, j - 1)];
                if (pt == 2) {
                    REAL e = w[0] * v[0] + w[1] * v[1] + w[2] * v[2];
                    U += (c->a[AIX(c, 0, i, j)] - (e + SC(c, i, j))) / T;
                }
                u[AIX(c, 0, i, j)] = U;
            }
            if (FN(nwa_lse3)(v[3], v[4], v[5], T) > (REAL)NEG_BIG) {
                FN(nwa_w3)(v[3], v[4], v[5], T, w);
                REAL U = w[0] * (u[AIX(c, 0, i - 1, j)] + dI[0]) + w[1] * (u[AIX(c, 1, i - 1, j)] + dI[1]) +
                         w[2] * (u[AIX(c, 2, i - 1, j)] + dI[2]);
                if (pt == 2) {
                    REAL e = w[0] * v[3] + w[1] * v[4] + w[2] * v[5];
                    U += (c->a[AIX(c, 1, i, j)] - e) / T;
                }
                u[AIX(c, 1, i, j)] = U;
            }
            if (FN(nwa_lse3)(v[6], v[7], v[8], T) > (REAL)NEG_BIG) {
                FN(nwa_w3)(v[6], v[7], v[8], T, w);
                REAL U = w[0] * (u[AIX(c, 0, i, j - 1)] + dD[0]) + w[1] * (u[AIX(c, 1, i, j - 1)] + dD[1]) +
                         w[2] * (u[AIX(c, 2, i, j - 1)] + dD[2]);
                if (pt == 2) {
                    REAL e = w[0] * v[6] + w[1] * v[7] + w[2] * v[8];
                    U += (c->a[AIX(c, 2, i, j)] - e) / T;
                }
                u[AIX(c, 2, i, j)] = U;
            }
        }
    }
    {
        size_t f[3] = {AIX(c, 0, c->L1, c->L2), AIX(c, 1, c->L1, c->L2), AIX(c, 2, c->L1, c->L2)};
        FN(nwa_w3)(c->a[f[0]], c->a[f[1]], c->a[f[2]], T, w);
        for (int st = 0; st < 3; ++st) { be[f[st]] = w[st]; t[st] = u[f[st]]; }
        FN(nwa_dw)(w, t, T, dw);
        if (pt == 2) {
            REAL e = w[0] * c->a[f[0]] + w[1] * c->a[f[1]] + w[2] * c->a[f[2]];
            REAL it2 = (REAL)1 / (T * T);
            for (int st = 0; st < 3; ++st) dw[st] += w[st] * (e - c->a[f[st]]) * it2;
        }
        for (int st = 0; st < 3; ++st) wt[f[st]] = dw[st];
    }
    NW_DIAGS(c, k, i, j) {
        REAL bM = be[AIX(c, 0, i, j)], bI = be[AIX(c, 1, i, j)], bD = be[AIX(c, 2, i, j)];
        REAL WM = wt[AIX(c, 0, i, j)], WI = wt[AIX(c, 1, i, j)], WD = wt[AIX(c, 2, i, j)];
        FN(nwa_cands)(c, c->a, i, j, v);
        REAL it2 = (REAL)1 / (T * T);
        if ((bM > NWA_TH || FABS(WM) > NWA_TH) && FN(nwa_lse3)(v[0], v[1], v[2], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[0], v[1], v[2], T, w);
            for (int st = 0; st < 3; ++st) t[st] = u[AIX(c, st, i - 1, j - 1)];
            FN(nwa_dw)(w, t, T, dw);
            if (pt == 2) {
                REAL e = w[0] * v[0] + w[1] * v[1] + w[2] * v[2];
                for (int st = 0; st < 3; ++st) dw[st] += w[st] * (e - v[st]) * it2;
            }
            for (int st = 0; st < 3; ++st)
                if (v[st] > (REAL)NEG_BIG) {
                    be[AIX(c, st, i - 1, j - 1)] += bM * w[st];
                    wt[AIX(c, st, i - 1, j - 1)] += WM * w[st] + bM * dw[st];
                }
            dP[(size_t)(i - 1) * c->ld + (j - 1)] += WM;
        }
        if ((bI > NWA_TH || FABS(WI) > NWA_TH) && FN(nwa_lse3)(v[3], v[4], v[5], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[3], v[4], v[5], T, w);
            for (int st = 0; st < 3; ++st) t[st] = u[AIX(c, st, i - 1, j)] + dI[st];
            FN(nwa_dw)(w, t, T, dw);
            if (pt == 2) {
                REAL e = w[0] * v[3] + w[1] * v[4] + w[2] * v[5];
                for (int st = 0; st < 3; ++st) dw[st] += w[st] * (e - v[3 + st]) * it2;
            }
            for (int st = 0; st < 3; ++st) {
                be[AIX(c, st, i - 1, j)] += bI * w[st];
                wt[AIX(c, st, i - 1, j)] += WI * w[st] + bI * dw[st];
            }
        }
        if ((bD > NWA_TH || FABS(WD) > NWA_TH) && FN(nwa_lse3)(v[6], v[7], v[8], T) > (REAL)NEG_BIG) {
            FN(nwa_w3)(v[6], v[7], v[8], T, w);
            for (int st = 0; st < 3; ++st) t[st] = u[AIX(c, st, i, j - 1)] + dD[st];
            FN(nwa_dw)(w, t, T, dw);
            if (pt == 2) {
                REAL e = w[0] * v[6] + w[1] * v[7] + w[2] * v[8];
                for (int st = 0; st < 3; ++st) dw[st] += w[st] * (e - v[6 + st]) * it2;
            }
            for (int st = 0; st < 3; ++st) {
                be[AIX(c, st, i, j - 1)] += bD * w[st];
                wt[AIX(c, st, i, j - 1)] += WD * w[st] + bD * dw[st];
            }
        }
    }
}

/* ---- Saigo-Vert local alignment (affine gaps; linear = go = ge = gap) ----
 * src/sv_affine/kernels_cpu.cpp and src/sv_linear/kernels_cpu.cpp: the local
 * affine model with one more transition, D <- I (gap open) from the left,
 * and S = LSE(0, M cells) -- only M states end an alignment, so only M has a
 * beta-init.  M's candidates add the score inside each term (diag + s and the
 * start term s), as the reference writes them.  `lin` selects the linear
 * file's accumulation of dS/dgap (one Kahan sum) and its gap direction (every
 * gap term). */

static void FN(sv_cands)(const FN(aff_t) *c, const REAL *t, int i, int j, REAL v[9]) {
    REAL s = SC(c, i, j);
    int dg = i > 1 && j > 1;
    v[0] = dg ? t[AIX(c, 0, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    v[1] = dg ? t[AIX(c, 1, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    v[2] = dg ? t[AIX(c, 2, i - 1, j - 1)] + s : (REAL)NEG_BIG;
    v[3] = s;
    v[4] = i > 1 ? t[AIX(c, 0, i - 1, j)] + c->go : (REAL)NEG_BIG;
    v[5] = i > 1 ? t[AIX(c, 1, i - 1, j)] + c->ge : (REAL)NEG_BIG;
    v[6] = j > 1 ? t[AIX(c, 0, i, j - 1)] + c->go : (REAL)NEG_BIG;
    v[7] = j > 1 ? t[AIX(c, 1, i, j - 1)] + c->go : (REAL)NEG_BIG;
    v[8] = j > 1 ? t[AIX(c, 2, i, j - 1)] + c->ge : (REAL)NEG_BIG;
}

/* src/sv_affine/kernels_cpu.cpp:81-196 */
static REAL FN(sv_forward)(FN(aff_t) *c) {
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) c->a[AIX(c, st, i, j)] = (REAL)NEG_BIG;
    c->a[AIX(c, 0, 0, 0)] = 0;
    REAL v[9];
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            FN(sv_cands)(c, c->a, i, j, v);
            c->a[AIX(c, 0, i, j)] = FN(tlse)(v, 4, c->T);
            c->a[AIX(c, 1, i, j)] = FN(tlse)(v + 4, 2, c->T);
            c->a[AIX(c, 2, i, j)] = FN(tlse)(v + 6, 3, c->T);
        }
    }
    REAL m = 0;   /* the empty alignment (score 0) */
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j)
            if (c->a[AIX(c, 0, i, j)] > m) m = c->a[AIX(c, 0, i, j)];
    FN(ksum_t) k = {0, 0};
    FN(kadd)(&k, FN(clip_exp)((0 - m) / c->T));
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            REAL x = c->a[AIX(c, 0, i, j)];
            if (x > (REAL)NEG_BIG) FN(kadd)(&k, FN(clip_exp)((x - m) / c->T));
        }
    return m + c->T * LOGF(k.s);
}

#define SV_LIVE(b) (!isinf(b) && !isnan(b) && (b) != 0)

/* src/sv_affine/kernels_cpu.cpp:200-365, src/sv_linear/kernels_cpu.cpp:207-370;
 * affine g = dS/d(go, ge, T); linear g[0] = dS/dgap, g[2] = dS/dT. */
static void FN(sv_adjoint)(const FN(aff_t) *c, REAL S, REAL *be, REAL *post, int L1max, int lin,
                           REAL g[3]) {
    size_t nsc = (size_t)L1max * c->ld;
    for (size_t q = 0; q < nsc; ++q) post[q] = 0;
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) be[AIX(c, st, i, j)] = 0;
    const REAL T = c->T;
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            REAL lp = (c->a[AIX(c, 0, i, j)] - S) / T;
            if (lp > 0) lp = 0;
            be[AIX(c, 0, i, j)] = FN(clip_exp)(lp);
        }
    REAL so = 0, se = 0, w[4], v[9];
    FN(ksum_t) gk = {0, 0};
    NW_DIAGS(c, k, i, j) {
        FN(sv_cands)(c, c->a, i, j, v);
        REAL bM = be[AIX(c, 0, i, j)];
        if (SV_LIVE(bM)) {
            FN(tsoftmax)(v, 4, T, w);
            post[(size_t)(i - 1) * c->ld + (j - 1)] += bM * (w[0] + w[1] + w[2] + w[3]);
            if (i > 1 && j > 1)
                for (int st = 0; st < 3; ++st)
                    if (w[st] > 0) be[AIX(c, st, i - 1, j - 1)] += bM * w[st];
        }
        REAL bI = be[AIX(c, 1, i, j)];
        if (SV_LIVE(bI)) {
            FN(tsoftmax)(v + 4, 2, T, w);
            if (i > 1) {
                if (w[0] > 0) {
                    be[AIX(c, 0, i - 1, j)] += bI * w[0];
                    if (lin) FN(kadd)(&gk, bI * w[0]); else so += bI * w[0];
                }
                if (w[1] > 0) {
                    be[AIX(c, 1, i - 1, j)] += bI * w[1];
                    if (lin) FN(kadd)(&gk, bI * w[1]); else se += bI * w[1];
                }
            }
        }
        REAL bD = be[AIX(c, 2, i, j)];
        if (SV_LIVE(bD)) {
            FN(tsoftmax)(v + 6, 3, T, w);
            if (j > 1) {
                if (w[0] > 0) {
                    be[AIX(c, 0, i, j - 1)] += bD * w[0];
                    if (lin) FN(kadd)(&gk, bD * w[0]); else so += bD * w[0];
                }
                if (w[1] > 0) {
                    be[AIX(c, 1, i, j - 1)] += bD * w[1];
                    if (lin) FN(kadd)(&gk, bD * w[1]); else so += bD * w[1];
                }
                if (w[2] > 0) {
                    be[AIX(c, 2, i, j - 1)] += bD * w[2];
                    if (lin) FN(kadd)(&gk, bD * w[2]); else se += bD * w[2];
                }
            }
        }
    }
    FN(ksum_t) ms = {0, 0};
    for (size_t q = 0; q < nsc; ++q) FN(kadd)(&ms, post[q] * c->s[q]);
    if (lin) {
        REAL gc = gk.s;
        FN(ksum_t) et = {0, 0};
        FN(kadd)(&et, ms.s);
        FN(kadd)(&et, gc * c->go);
        g[0] = gc; g[1] = 0; g[2] = (S - et.s) / T;
    } else {
        REAL egc = so * c->go + se * c->ge;
        REAL et = ms.s + egc;
        g[0] = so; g[1] = se; g[2] = (S - et) / T;
    }
}

/* src/sv_affine/kernels_cpu.cpp:369-620 (HVP; the linear file's is the same). */
static void FN(sv_hvp)(FN(aff_t) *c, REAL S, const REAL *V, REAL *da, REAL *dbe, REAL *be,
                       REAL *H, int L1max) {
    size_t nsc = (size_t)L1max * c->ld;
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) {
                size_t o = AIX(c, st, i, j);
                da[o] = 0; dbe[o] = 0; be[o] = 0;
            }
    for (size_t q = 0; q < nsc; ++q) H[q] = 0;
    const REAL T = c->T;
    REAL w[4], v[9], t[4], dw[4];
#define VV(i, j) V[(size_t)((i) - 1) * c->ld + (size_t)((j) - 1)]
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            REAL vv = VV(i, j);
            int dg = i > 1 && j > 1;
            FN(sv_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 4, T, w);
            for (int st = 0; st < 3; ++st) t[st] = dg ? da[AIX(c, st, i - 1, j - 1)] + vv : 0;
            t[3] = vv;
            da[AIX(c, 0, i, j)] = w[0] * t[0] + w[1] * t[1] + w[2] * t[2] + w[3] * t[3];
            FN(tsoftmax)(v + 4, 2, T, w);
            da[AIX(c, 1, i, j)] = w[0] * (i > 1 ? da[AIX(c, 0, i - 1, j)] : 0) +
                                  w[1] * (i > 1 ? da[AIX(c, 1, i - 1, j)] : 0);
            FN(tsoftmax)(v + 6, 3, T, w);
            da[AIX(c, 2, i, j)] = w[0] * (j > 1 ? da[AIX(c, 0, i, j - 1)] : 0) +
                                  w[1] * (j > 1 ? da[AIX(c, 1, i, j - 1)] : 0) +
                                  w[2] * (j > 1 ? da[AIX(c, 2, i, j - 1)] : 0);
        }
    }
    FN(ksum_t) dk = {0, 0};
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j)
            FN(kadd)(&dk, FN(end_weight)(c->a[AIX(c, 0, i, j)], S, T) * da[AIX(c, 0, i, j)]);
    REAL dS = dk.s;
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) be[AIX(c, 0, i, j)] = FN(end_weight)(c->a[AIX(c, 0, i, j)], S, T);
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) {
            size_t o = AIX(c, 0, i, j);
            dbe[o] = be[o] * (da[o] - dS) / T;
        }
    NW_DIAGS(c, k, i, j) {
        REAL vv = VV(i, j);
        int dg = i > 1 && j > 1;
        FN(sv_cands)(c, c->a, i, j, v);
        REAL bM = be[AIX(c, 0, i, j)], dM = dbe[AIX(c, 0, i, j)];
        FN(tsoftmax)(v, 4, T, w);
        for (int st = 0; st < 3; ++st) t[st] = dg ? da[AIX(c, st, i - 1, j - 1)] + vv : 0;
        t[3] = vv;
        REAL e = w[0] * t[0] + w[1] * t[1] + w[2] * t[2] + w[3] * t[3];
        for (int q = 0; q < 4; ++q) dw[q] = w[q] * (t[q] - e) / T;
        H[(size_t)(i - 1) * c->ld + (j - 1)] += dM * (w[0] + w[1] + w[2] + w[3]) +
                                                bM * (dw[0] + dw[1] + dw[2] + dw[3]);
        if (dg)
            for (int st = 0; st < 3; ++st) be[AIX(c, st, i - 1, j - 1)] += bM * w[st];
        if (dg)
            for (int st = 0; st < 3; ++st)
                dbe[AIX(c, st, i - 1, j - 1)] += dM * w[st] + bM * dw[st];
        REAL bI = be[AIX(c, 1, i, j)], dI = dbe[AIX(c, 1, i, j)];
        FN(tsoftmax)(v + 4, 2, T, w);
        t[0] = i > 1 ? da[AIX(c, 0, i - 1, j)] : 0;
        t[1] = i > 1 ? da[AIX(c, 1, i - 1, j)] : 0;
        e = w[0] * t[0] + w[1] * t[1];
        dw[0] = w[0] * (t[0] - e) / T;
        dw[1] = w[1] * (t[1] - e) / T;
        if (i > 1) {
            be[AIX(c, 0, i - 1, j)] += bI * w[0];
            be[AIX(c, 1, i - 1, j)] += bI * w[1];
        }
        if (i > 1) {
            dbe[AIX(c, 0, i - 1, j)] += dI * w[0] + bI * dw[0];
            dbe[AIX(c, 1, i - 1, j)] += dI * w[1] + bI * dw[1];
        }
        REAL bD = be[AIX(c, 2, i, j)], dD = dbe[AIX(c, 2, i, j)];
        FN(tsoftmax)(v + 6, 3, T, w);
        for (int st = 0; st < 3; ++st) t[st] = j > 1 ? da[AIX(c, st, i, j - 1)] : 0;
        e = w[0] * t[0] + w[1] * t[1] + w[2] * t[2];
        for (int q = 0; q < 3; ++q) dw[q] = w[q] * (t[q] - e) / T;
        if (j > 1)
            for (int st = 0; st < 3; ++st) be[AIX(c, st, i, j - 1)] += bD * w[st];
        if (j > 1)
            for (int st = 0; st < 3; ++st) dbe[AIX(c, st, i, j - 1)] += dD * w[st] + bD * dw[st];
    }
#undef VV
}

/* src/sv_affine/kernels_cpu.cpp:630-934 (dP/dtheta); pt 0 = gap_open, 1 =
 * gap_ext, 2 = temperature, 3 = the linear model's single gap (every gap term). */
static void FN(sv_param)(FN(aff_t) *c, REAL S, REAL dSdt, int pt, REAL *u, REAL *be, REAL *wt,
                         REAL *dP, int L1max) {
    size_t nsc = (size_t)L1max * c->ld;
    for (int st = 0; st < 3; ++st)
        for (int i = 0; i <= c->L1; ++i)
            for (int j = 0; j <= c->L2; ++j) {
                size_t o = AIX(c, st, i, j);
                u[o] = 0; be[o] = 0; wt[o] = 0;
            }
    for (size_t q = 0; q < nsc; ++q) dP[q] = 0;
    const REAL T = c->T;
    const int TM = pt == 2;
    /* direct tangents: I <- (M open, I ext); D <- (M open, I open, D ext) */
    const REAL dI[2] = {(pt == 0 || pt == 3) ? 1 : 0, (pt == 1 || pt == 3) ? 1 : 0};
    const REAL dD[3] = {(pt == 0 || pt == 3) ? 1 : 0, (pt == 0 || pt == 3) ? 1 : 0,
                        (pt == 1 || pt == 3) ? 1 : 0};
    REAL w[4], v[9], t[4], dw[4];
    for (int k = 2; k <= c->L1 + c->L2; ++k) {
        int i0 = (k - c->L2 > 1) ? k - c->L2 : 1;
        int i1 = (c->L1 < k - 1) ? c->L1 : k - 1;
        for (int i = i0; i <= i1; ++i) {
            int j = k - i;
            int dg = i > 1 && j > 1;
            FN(sv_cands)(c, c->a, i, j, v);
            FN(tsoftmax)(v, 4, T, w);
            REAL U = w[0] * (dg ? u[AIX(c, 0, i - 1, j - 1)] : 0) + w[1] * (dg ? u[AIX(c, 1, i - 1, j - 1)] : 0) +
                     w[2] * (dg ? u[AIX(c, 2, i - 1, j - 1)] : 0);
            if (TM) {
                REAL e = w[0] * v[0] + w[1] * v[1] + w[2] * v[2] + w[3] * v[3];
                U += (c->a[AIX(c, 0, i, j)] - e) / T;
            }
            u[AIX(c, 0, i, j)] = U;
            FN(tsoftmax)(v + 4, 2, T, w);
            t[0] = (i > 1 ? u[AIX(c, 0, i - 1, j)] : 0) + dI[0];
            t[1] = (i > 1 ? u[AIX(c, 1, i - 1, j)] : 0) + dI[1];
            U = w[0] * t[0] + w[1] * t[1];
            if (TM) {
                REAL e = w[0] * v[4] + w[1] * v[5];
                U += (c->a[AIX(c, 1, i, j)] - e) / T;
            }
            u[AIX(c, 1, i, j)] = U;
            FN(tsoftmax)(v + 6, 3, T, w);
            for (int st = 0; st < 3; ++st) t[st] = (j > 1 ? u[AIX(c, st, i, j - 1)] : 0) + dD[st];
            U = w[0] * t[0] + w[1] * t[1] + w[2] * t[2];
            if (TM) {
                REAL e = w[0] * v[6] + w[1] * v[7] + w[2] * v[8];
                U += (c->a[AIX(c, 2, i, j)] - e) / T;
            }
            u[AIX(c, 2, i, j)] = U;
        }
    }
    for (int i = 1; i <= c->L1; ++i)
        for (int j = 1; j <= c->L2; ++j) be[AIX(c, 0, i, j)] = FN(end_weight)(c->a[AIX(c, 0, i, j)], S, T);
    REAL it2 = (REAL)1 / (T * T);
    NW_DIAGS(c, k, i, j) {
        int dg = i > 1 && j > 1;
        size_t oM = AIX(c, 0, i, j), oI = AIX(c, 1, i, j), oD = AIX(c, 2, i, j);
        FN(sv_cands)(c, c->a, i, j, v);
        REAL bM = be[oM];
        REAL b0 = FN(end_weight)(c->a[oM], S, T);
        REAL WM = wt[oM] + b0 * (u[oM] - dSdt) / T;
        if (TM && c->a[oM] > (REAL)NEG_BIG) WM -= b0 * (c->a[oM] - S) / (T * T);
        FN(tsoftmax)(v, 4, T, w);
        for (int st = 0; st < 3; ++st) t[st] = dg ? u[AIX(c, st, i - 1, j - 1)] : 0;
        t[3] = 0;
        REAL e = w[0] * t[0] + w[1] * t[1] + w[2] * t[2] + w[3] * t[3];
        for (int q = 0; q < 4; ++q) dw[q] = w[q] * (t[q] - e) / T;
        if (TM) {
            REAL ev = w[0] * v[0] + w[1] * v[1] + w[2] * v[2] + w[3] * v[3];
            for (int q = 0; q < 4; ++q) dw[q] += w[q] * (ev - v[q]) * it2;
        }
        dP[(size_t)(i - 1) * c->ld + (j - 1)] += WM;
        if (dg)
            for (int st = 0; st < 3; ++st) {
                be[AIX(c, st, i - 1, j - 1)] += bM * w[st];
                wt[AIX(c, st, i - 1, j - 1)] += WM * w[st] + bM * dw[st];
            }
        REAL bI = be[oI], WI = wt[oI];
        if (i > 1) {
            FN(tsoftmax)(v + 4, 2, T, w);
            t[0] = u[AIX(c, 0, i - 1, j)] + dI[0];
            t[1] = u[AIX(c, 1, i - 1, j)] + dI[1];
            e = w[0] * t[0] + w[1] * t[1];
            dw[0] = w[0] * (t[0] - e) / T;
            dw[1] = w[1] * (t[1] - e) / T;
            if (TM) {
                REAL ev = w[0] * v[4] + w[1] * v[5];
                dw[0] += w[0] * (ev - v[4]) * it2;
                dw[1] += w[1] * (ev - v[5]) * it2;
            }
            for (int st = 0; st < 2; ++st) {
                be[AIX(c, st, i - 1, j)] += bI * w[st];
                wt[AIX(c, st, i - 1, j)] += WI * w[st] + bI * dw[st];
            }
        }
        REAL bD = be[oD], WD = wt[oD];
        if (j > 1) {
            FN(tsoftmax)(v + 6, 3, T, w);
            for (int st = 0; st < 3; ++st) t[st] = u[AIX(c, st, i, j - 1)] + dD[st];
            e = w[0] * t[0] + w[1] * t[1] + w[2] * t[2];
            for (int q = 0; q < 3; ++q) dw[q] = w[q] * (t[q] - e) / T;
            if (TM) {
                REAL ev = w[0] * v[6] + w[1] * v[7] + w[2] * v[8];
                for (int q = 0; q < 3; ++q) dw[q] += w[q] * (ev - v[6 + q]) * it2;
            }
            for (int st = 0; st < 3; ++st) {
                be[AIX(c, st, i, j - 1)] += bD * w[st];
                wt[AIX(c, st, i, j - 1)] += WD * w[st] + bD * dw[st];
            }
        }
    }
}

/* ---- batched entry points (padded [B, L1max, L2max] layout) ------------ */

static int FN(pair_len)(const int *lengths, int b, int which, int dflt) {
    return lengths ? lengths[2 * b + which] : dflt;
}

/* value + map + dS/d(go, ge, T), like orihime::sw_affine_forward plus
 * value_grad_params.  grads may be NULL. */
int FN(oracle_sw_affine_forward)(const REAL *scores, const int *lengths, int B, int L1m,
                                 int L2m, REAL go, REAL ge, REAL T, REAL *value, REAL *map,
                                 REAL *gopen, REAL *gext, REAL *gT) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 3 * plane);
    REAL *be = (REAL *)malloc(sizeof(REAL) * 3 * plane);
    if (!a || !be) { free(a); free(be); return -1; }
    for (int b = 0; b < B; ++b) {
        FN(aff_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.go = go; c.ge = ge; c.T = T;
        c.plane = plane; c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(aff_forward)(&c);
        REAL g[3];
        FN(aff_adjoint)(&c, S, be, map + b * slab, L1m, g);
        value[b] = S;
        if (gopen) gopen[b] = g[0];
        if (gext) gext[b] = g[1];
        if (gT) gT[b] = g[2];
    }
    free(a); free(be);
    return 0;
}

int FN(oracle_sw_affine_hvp)(const REAL *scores, const REAL *V, const int *lengths, int B,
                             int L1m, int L2m, REAL go, REAL ge, REAL T, REAL *out) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *buf = (REAL *)malloc(sizeof(REAL) * 12 * plane);
    if (!buf) return -1;
    REAL *a = buf, *be = buf + 3 * plane, *da = buf + 6 * plane, *dbe = buf + 9 * plane;
    for (int b = 0; b < B; ++b) {
        FN(aff_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.go = go; c.ge = ge; c.T = T;
        c.plane = plane; c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(aff_forward)(&c);
        FN(aff_hvp)(&c, S, V + b * slab, da, be, dbe, out + b * slab, L1m);
    }
    free(buf);
    return 0;
}

/* pt: 0 = gap_open, 1 = gap_ext, 2 = temperature. */
int FN(oracle_sw_affine_param_grad)(const REAL *scores, const int *lengths, int B, int L1m,
                                    int L2m, REAL go, REAL ge, REAL T, int pt, REAL *out) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *buf = (REAL *)malloc(sizeof(REAL) * (15 * plane + slab));
    if (!buf) return -1;
    REAL *a = buf, *be = buf + 3 * plane, *u = buf + 6 * plane, *w = buf + 9 * plane;
    REAL *be2 = buf + 12 * plane, *post = buf + 15 * plane;
    for (int b = 0; b < B; ++b) {
        FN(aff_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.go = go; c.ge = ge; c.T = T;
        c.plane = plane; c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(aff_forward)(&c);
        REAL g[3];
        FN(aff_adjoint)(&c, S, be2, post, L1m, g);
        FN(aff_param)(&c, S, g[pt], pt, u, be, w, out + b * slab, L1m);
    }
    free(buf);
    return 0;
}

int FN(oracle_sw_linear_forward)(const REAL *scores, const int *lengths, int B, int L1m,
                                 int L2m, REAL gap, REAL T, REAL *value, REAL *map,
                                 REAL *ggap, REAL *gT) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 2 * plane);
    if (!a) return -1;
    REAL *be = a + plane;
    for (int b = 0; b < B; ++b) {
        FN(lin_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.g = gap; c.T = T;
        c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(lin_forward)(&c);
        REAL g[2];
        FN(lin_adjoint)(&c, S, be, map + b * slab, L1m, g);
        value[b] = S;
        if (ggap) ggap[b] = g[0];
        if (gT) gT[b] = g[1];
    }
    free(a);
    return 0;
}

int FN(oracle_sw_linear_hvp)(const REAL *scores, const REAL *V, const int *lengths, int B,
                             int L1m, int L2m, REAL gap, REAL T, REAL *out) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *buf = (REAL *)malloc(sizeof(REAL) * 4 * plane);
    if (!buf) return -1;
    REAL *a = buf, *be = buf + plane, *da = buf + 2 * plane, *dbe = buf + 3 * plane;
    for (int b = 0; b < B; ++b) {
        FN(lin_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.g = gap; c.T = T;
        c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(lin_forward)(&c);
        FN(lin_hvp)(&c, S, V + b * slab, da, be, dbe, out + b * slab, L1m);
    }
    free(buf);
    return 0;
}

/* pt: 0 = gap, 1 = temperature. */
int FN(oracle_sw_linear_param_grad)(const REAL *scores, const int *lengths, int B, int L1m,
                                    int L2m, REAL gap, REAL T, int pt, REAL *out) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *buf = (REAL *)malloc(sizeof(REAL) * (5 * plane + slab));
    if (!buf) return -1;
    REAL *a = buf, *be = buf + plane, *u = buf + 2 * plane, *w = buf + 3 * plane;
    REAL *be2 = buf + 4 * plane, *post = buf + 5 * plane;
    for (int b = 0; b < B; ++b) {
        FN(lin_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.g = gap; c.T = T;
        c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(lin_forward)(&c);
        REAL g[2];
        FN(lin_adjoint)(&c, S, be2, post, L1m, g);
        FN(lin_param)(&c, S, g[pt], pt, u, be, w, out + b * slab, L1m);
    }
    free(buf);
    return 0;
}

int FN(oracle_nw_linear_forward)(const REAL *scores, const int *lengths, int B, int L1m,
                                 int L2m, REAL gap, REAL T, REAL *value, REAL *map,
                                 REAL *ggap, REAL *gT) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 2 * plane);
    if (!a) return -1;
    REAL *be = a + plane;
    for (int b = 0; b < B; ++b) {
        FN(lin_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.g = gap; c.T = T;
        c.cols = (size_t)L2m + 1; c.a = a;
        REAL S = FN(nw_forward)(&c);
        REAL g[2];
        FN(nw_adjoint)(&c, S, be, map + b * slab, L1m, g);
        value[b] = S;
        if (ggap) ggap[b] = g[0];
        if (gT) gT[b] = g[1];
    }
    free(a);
    return 0;
}

int FN(oracle_nw_linear_hvp)(const REAL *scores, const REAL *V, const int *lengths, int B,
                             int L1m, int L2m, REAL gap, REAL T, REAL *out) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *buf = (REAL *)malloc(sizeof(REAL) * 4 * plane);
    if (!buf) return -1;
    REAL *a = buf, *be = buf + plane, *da = buf + 2 * plane, *dbe = buf + 3 * plane;
    for (int b = 0; b < B; ++b) {
        FN(lin_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.g = gap; c.T = T;
        c.cols = (size_t)L2m + 1; c.a = a;
        FN(nw_forward)(&c);
        FN(nw_hvp)(&c, V + b * slab, da, be, dbe, out + b * slab, L1m);
    }
    free(buf);
    return 0;
}

/* pt: 0 = gap, 1 = temperature. */
int FN(oracle_nw_linear_param_grad)(const REAL *scores, const int *lengths, int B, int L1m,
                                    int L2m, REAL gap, REAL T, int pt, REAL *out) {
    size_t slab = (size_t)L1m * L2m;
    size_t plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *buf = (REAL *)malloc(sizeof(REAL) * 4 * plane);
    if (!buf) return -1;
    REAL *a = buf, *be = buf + plane, *u = buf + 2 * plane, *w = buf + 3 * plane;
    for (int b = 0; b < B; ++b) {
        FN(lin_t) c;
        c.L1 = FN(pair_len)(lengths, b, 0, L1m);
        c.L2 = FN(pair_len)(lengths, b, 1, L2m);
        c.ld = L2m; c.s = scores + b * slab; c.g = gap; c.T = T;
        c.cols = (size_t)L2m + 1; c.a = a;
        FN(nw_forward)(&c);
        FN(nw_param)(&c, pt, u, be, w, out + b * slab, L1m);
    }
    free(buf);
    return 0;
}

#define NWA_PAIR()                                                            \
    FN(aff_t) c;                                                              \
    c.L1 = FN(pair_len)(lengths, b, 0, L1m);                                  \
    c.L2 = FN(pair_len)(lengths, b, 1, L2m);                                  \
    c.ld = L2m; c.s = scores + b * slab; c.go = go; c.ge = ge; c.T = T;       \
    c.plane = plane; c.cols = (size_t)L2m + 1; c.a = a

int FN(oracle_nw_affine_forward)(const REAL *scores, const int *lengths, int B, int L1m, int L2m,
                                 REAL go, REAL ge, REAL T, REAL *value, REAL *map, REAL *gopen,
                                 REAL *gext, REAL *gT) {
    size_t slab = (size_t)L1m * L2m, plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 6 * plane);
    if (!a) return -1;
    REAL *be = a + 3 * plane;
    for (int b = 0; b < B; ++b) {
        NWA_PAIR();
        REAL S = FN(nwa_forward)(&c);
        REAL g[3];
        FN(nwa_adjoint)(&c, S, be, map + b * slab, L1m, g);
        value[b] = S;
        if (gopen) gopen[b] = g[0];
        if (gext) gext[b] = g[1];
        if (gT) gT[b] = g[2];
    }
    free(a);
    return 0;
}

int FN(oracle_nw_affine_hvp)(const REAL *scores, const REAL *V, const int *lengths, int B, int L1m,
                             int L2m, REAL go, REAL ge, REAL T, REAL *out) {
    size_t slab = (size_t)L1m * L2m, plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 12 * plane);
    if (!a) return -1;
    for (int b = 0; b < B; ++b) {
        NWA_PAIR();
        FN(nwa_forward)(&c);
        FN(nwa_hvp)(&c, V + b * slab, a + 3 * plane, a + 6 * plane, a + 9 * plane, out + b * slab, L1m);
    }
    free(a);
    return 0;
}

/* pt: 0 = gap_open, 1 = gap_ext, 2 = temperature. */
int FN(oracle_nw_affine_param_grad)(const REAL *scores, const int *lengths, int B, int L1m,
                                    int L2m, REAL go, REAL ge, REAL T, int pt, REAL *out) {
    size_t slab = (size_t)L1m * L2m, plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 12 * plane);
    if (!a) return -1;
    for (int b = 0; b < B; ++b) {
        NWA_PAIR();
        FN(nwa_forward)(&c);
        FN(nwa_param)(&c, pt, a + 3 * plane, a + 6 * plane, a + 9 * plane, out + b * slab, L1m);
    }
    free(a);
    return 0;
}

/* Saigo-Vert: lin = 0 affine (go, ge), 1 linear (go = ge = gap; grads in
 * gopen and gT, gext set to 0). */
int FN(oracle_sv_forward)(const REAL *scores, const int *lengths, int B, int L1m, int L2m, REAL go,
                          REAL ge, REAL T, int lin, REAL *value, REAL *map, REAL *gopen,
                          REAL *gext, REAL *gT) {
    size_t slab = (size_t)L1m * L2m, plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 6 * plane);
    if (!a) return -1;
    for (int b = 0; b < B; ++b) {
        NWA_PAIR();
        REAL S = FN(sv_forward)(&c);
        REAL g[3];
        FN(sv_adjoint)(&c, S, a + 3 * plane, map + b * slab, L1m, lin, g);
        value[b] = S;
        if (gopen) gopen[b] = g[0];
        if (gext) gext[b] = g[1];
        if (gT) gT[b] = g[2];
    }
    free(a);
    return 0;
}

int FN(oracle_sv_hvp)(const REAL *scores, const REAL *V, const int *lengths, int B, int L1m,
                      int L2m, REAL go, REAL ge, REAL T, REAL *out) {
    size_t slab = (size_t)L1m * L2m, plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 12 * plane);
    if (!a) return -1;
    for (int b = 0; b < B; ++b) {
        NWA_PAIR();
        REAL S = FN(sv_forward)(&c);
        FN(sv_hvp)(&c, S, V + b * slab, a + 3 * plane, a + 6 * plane, a + 9 * plane, out + b * slab, L1m);
    }
    free(a);
    return 0;
}

/* pt: 0 = gap_open, 1 = gap_ext, 2 = temperature, 3 = linear gap. */
int FN(oracle_sv_param_grad)(const REAL *scores, const int *lengths, int B, int L1m, int L2m,
                             REAL go, REAL ge, REAL T, int lin, int pt, REAL *out) {
    size_t slab = (size_t)L1m * L2m, plane = (size_t)(L1m + 1) * (L2m + 1);
    REAL *a = (REAL *)malloc(sizeof(REAL) * 15 * plane + sizeof(REAL) * slab);
    if (!a) return -1;
    REAL *post = a + 15 * plane;
    for (int b = 0; b < B; ++b) {
        NWA_PAIR();
        REAL S = FN(sv_forward)(&c);
        REAL g[3];
        FN(sv_adjoint)(&c, S, a + 12 * plane, post, L1m, lin, g);
        REAL dS = pt == 2 ? g[2] : (pt == 1 ? g[1] : g[0]);
        FN(sv_param)(&c, S, dS, pt, a + 3 * plane, a + 6 * plane, a + 9 * plane, out + b * slab, L1m);
    }
    free(a);
    return 0;
}

#undef SV_LIVE
#undef NWA_PAIR
#undef NWA_TH
#undef NW_DIAGS
#undef AIX
#undef SC
#undef LIX
#undef FN
#undef CAT
#undef CAT2
