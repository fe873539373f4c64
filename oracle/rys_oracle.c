/*
 * ORACLE -- test infrastructure only.  Nothing in the product path links or
 * calls this file; only tests/, the smoke check and the CPU-baseline leg of
 * bench.py load it, and only as the checker.
 *
 * CPU restatement of the reference's Rys-quadrature DF integrals over
 * Cartesian Gaussian shells (asuka/cueri/_eri_rys_cpu.pyx):
 *
 *   boys_list        <- _boys_fm_list                (_eri_rys_cpu.pyx:194-216)
 *   rys_roots        <- _rys_roots_weights_generic   (_eri_rys_cpu.pyx:547-658)
 *                       + _tridiag_eigh_ql           (_eri_rys_cpu.pyx:441-544)
 *   compute_G        <- _compute_G                   (_eri_rys_cpu.pyx:690-718)
 *   shift_ld0        <- _shift_from_G_ld0_d          (_eri_rys_cpu.pyx:802-817)
 *   oracle_tile_3c   <- _eri_rys_tile_cart_kernel with the dummy s shell
 *                       (_eri_rys_cpu.pyx:880-1096; dummy: cueri_df_cpu.py:44-185)
 *   oracle_deriv_3c  <- df_int3c2e_deriv_contracted_cart_sp_cy (_eri_rys_cpu.pyx:2650-2957)
 *   oracle_deriv_2c  <- df_metric_2c2e_deriv_contracted_cart_sp_cy (_eri_rys_cpu.pyx:3750-4006)
 *
 * One deliberate difference: the Boys moments, the monomial Stieltjes
 * procedure and the QL eigensolve run in __float128 instead of double.  The
 * reference's double-precision version loses accuracy quickly with the root
 * count (about 7e-9 relative at 7 roots, 2e-6 at 9, 4e-4 at 10); in quad
 * precision the same steps are accurate to ~1e-16 for every root count used
 * here, so this oracle states what the reference's algorithm computes in
 * exact arithmetic.  All integral arithmetic after the roots is double, in
 * the reference's order.
 */
#include <math.h>
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>

typedef __float128 qd;

#define LMAX 8
#define LMAX_D (LMAX + 1)
#define STRIDE (2 * LMAX_D + 1)
#define NCART_MAX ((LMAX + 1) * (LMAX + 2) / 2)
#define NROOTS_MAX (LMAX + LMAX + 2)

static const double kPi = 3.141592653589793238462643383279502884;
static const double kTwoPi52 = 2.0 * 3.141592653589793238462643383279502884 * 3.141592653589793238462643383279502884 *
                               1.772453850905516027298167483341145182;

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void fill_cart(int l, int *lx, int *ly, int *lz) {
    int idx = 0;
    for (int x = l; x >= 0; --x)
        for (int y = l - x; y >= 0; --y) {
            lx[idx] = x;
            ly[idx] = y;
            lz[idx] = l - x - y;
            ++idx;
        }
}

/* ---- Boys function F_0..F_mmax (reference branches, quad precision) ---- */
static void boys_list(qd T, int mmax, qd *out) {
    const qd pi = M_PIq;
    if (T < 5) {
        qd term = 1, F = 0;
        for (int k = 0; k < 160; ++k) {
            F += term / (qd)(2 * mmax + 2 * k + 1);
            term *= -T / (qd)(k + 1);
        }
        out[mmax] = F;
        qd e = expq(-T);
        for (int m = mmax; m > 0; --m) out[m - 1] = (2 * T * out[m] + e) / (qd)(2 * m - 1);
        return;
    }
    out[0] = sqrtq(pi / T) * erfq(sqrtq(T)) / 2;
    qd e = expq(-T);
    for (int m = 1; m <= mmax; ++m) out[m] = ((qd)(2 * m - 1) * out[m - 1] - e) / (2 * T);
}

static qd poly_inner(const qd *a, int da, const qd *b, int db, const qd *mu, int shift) {
    qd s = 0;
    for (int i = 0; i <= da; ++i)
        for (int j = 0; j <= db; ++j) s += a[i] * b[j] * mu[i + j + shift];
    return s;
}

static void tridiag_ql(int n, qd *d, qd *e, qd *z0) {
    const qd eps = 1e-33Q;
    e[n - 1] = 0;
    for (int i = 0; i < n; ++i) z0[i] = (i == 0) ? 1 : 0;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        for (;;) {
            int m;
            for (m = l; m < n - 1; ++m) {
                qd dd = fabsq(d[m]) + fabsq(d[m + 1]);
                if (dd == 0) dd = 1;
                if (fabsq(e[m]) <= eps * dd) break;
            }
            if (m == l || iter >= 200) break;
            ++iter;
            qd g = (d[l + 1] - d[l]) / (2 * e[l]);
            qd r = sqrtq(g * g + 1);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? fabsq(r) : -fabsq(r)));
            qd s = 1, c = 1, p = 0;
            int cont = 0;
            for (int i = m - 1; i >= l; --i) {
                qd f = s * e[i], b = c * e[i];
                r = sqrtq(f * f + g * g);
                e[i + 1] = r;
                if (r == 0) {
                    d[i + 1] -= p;
                    e[m] = 0;
                    cont = 1;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                qd rr = (d[i] - g) * s + 2 * c * b;
                p = s * rr;
                d[i + 1] = g + p;
                g = c * rr - b;
                qd zi1 = z0[i + 1], zi = z0[i];
                z0[i + 1] = s * zi + c * zi1;
                z0[i] = c * zi - s * zi1;
            }
            if (cont) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0;
        }
    }
    for (int i = 0; i < n - 1; ++i) {
        int k = i;
        qd p = d[i];
        for (int j = i + 1; j < n; ++j)
            if (d[j] < p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            qd t = d[i];
            d[i] = d[k];
            d[k] = t;
            t = z0[i];
            z0[i] = z0[k];
            z0[k] = t;
        }
    }
}

/* Rys nodes (in x = t^2) and weights, ascending nodes. */
void oracle_rys_roots(int n, double Td, double *r, double *w) {
    qd mu[2 * NROOTS_MAX + 2], alpha[NROOTS_MAX + 1], beta[NROOTS_MAX + 1];
    qd pp[NROOTS_MAX + 2], pc[NROOTS_MAX + 2], pn[NROOTS_MAX + 2];
    qd d[NROOTS_MAX + 1], e[NROOTS_MAX + 1], z0[NROOTS_MAX + 1];
    qd T = (qd)Td;
    boys_list(T, 2 * n - 1, mu);
    qd mu0 = mu[0];
    for (int i = 0; i <= n; ++i) pp[i] = pc[i] = pn[i] = 0;
    pc[0] = 1;
    qd h = mu0;
    alpha[0] = mu[1] / mu0;
    beta[0] = 0;
    for (int k = 0; k < n - 1; ++k) {
        qd bk = (k >= 1 && h > 0) ? beta[k] : 0;
        for (int i = 0; i <= n; ++i) pn[i] = 0;
        for (int i = 0; i <= k; ++i) {
            pn[i + 1] += pc[i];
            pn[i] -= alpha[k] * pc[i];
        }
        if (k >= 1)
            for (int i = 0; i < k; ++i) pn[i] -= bk * pp[i];
        qd hn = poly_inner(pn, k + 1, pn, k + 1, mu, 0);
        if (hn < 0) hn = 0;
        beta[k + 1] = h > 0 ? hn / h : 0;
        qd an = poly_inner(pn, k + 1, pn, k + 1, mu, 1);
        alpha[k + 1] = hn > 0 ? an / hn : alpha[k];
        for (int i = 0; i <= n; ++i) {
            pp[i] = pc[i];
            pc[i] = pn[i];
        }
        h = hn;
    }
    for (int i = 0; i < n; ++i) {
        d[i] = alpha[i];
        e[i] = 0;
    }
    for (int i = 0; i < n - 1; ++i) e[i] = beta[i + 1] > 0 ? sqrtq(beta[i + 1]) : 0;
    tridiag_ql(n, d, e, z0);
    for (int i = 0; i < n; ++i) {
        qd x = d[i];
        if (x < 0) x = 0;
        if (x > 1) x = 1;
        r[i] = (double)x;
        w[i] = (double)(mu0 * z0[i] * z0[i]);
    }
}

void oracle_boys(double T, int mmax, double *out) {
    qd tmp[64];
    boys_list((qd)T, mmax, tmp);
    for (int m = 0; m <= mmax; ++m) out[m] = (double)tmp[m];
}

/* ---- 2D Rys recurrences and the horizontal shift (double) ---- */
static void compute_G(double *G, int nmax, int mmax, double C, double Cp, double B0, double B1, double B1p) {
    G[0] = 1.0;
    if (nmax > 0) G[1 * STRIDE] = C;
    if (mmax > 0) G[1] = Cp;
    for (int a = 2; a <= nmax; ++a) G[a * STRIDE] = B1 * (a - 1) * G[(a - 2) * STRIDE] + C * G[(a - 1) * STRIDE];
    for (int b = 2; b <= mmax; ++b) G[b] = B1p * (b - 1) * G[b - 2] + Cp * G[b - 1];
    if (mmax == 0 || nmax == 0) return;
    for (int a = 1; a <= nmax; ++a) {
        G[a * STRIDE + 1] = a * B0 * G[(a - 1) * STRIDE] + Cp * G[a * STRIDE];
        for (int b = 2; b <= mmax; ++b)
            G[a * STRIDE + b] = B1p * (b - 1) * G[a * STRIDE + b - 2] + a * B0 * G[(a - 1) * STRIDE + b - 1] +
                                Cp * G[a * STRIDE + b - 1];
    }
}

static double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double out = 1.0;
    int kk = k > n - k ? n - k : k;
    for (int i = 1; i <= kk; ++i) out *= (double)(n - kk + i) / (double)i;
    return out;
}

static double shift_ld0(const double *G, int i, int j, int k, const double *xij) {
    double out = 0.0;
    for (int n = 0; n <= j; ++n) out += binom(j, n) * xij[j - n] * G[(n + i) * STRIDE + k];
    return out;
}

/* Basis view: combined arrays with explicit centre/l/prims per shell. */
typedef struct {
    const double *cxyz;
    const int *l;
    const int *pstart;
    const int *nprim;
    const double *pexp;
    const double *pcoef;
} basis_t;

/* Per-primitive-triplet Rys setup for (A B | C dummy). Calls fn for each root. */
typedef struct {
    double A[3], B[3], C[3];
    double AB[3];
} geom_t;

/*
 * (A B | C) tile for one AO shell pair (A,B) and one aux shell C, with the
 * dummy s shell (exp 0, coef 1, at the origin) as D.  out[(ia*nB+ib)*nC+ic].
 * With B = dummy as well this is the metric tile (A | C).
 */
static void tile_3c(const basis_t *ao, int shA, int shB, int b_is_dummy, const basis_t *aux, int shC, double *out) {
    int la = ao->l[shA], lb = b_is_dummy ? 0 : ao->l[shB], lc = aux->l[shC];
    int nA = ncart(la), nB = ncart(lb), nC = ncart(lc);
    int Alx[NCART_MAX], Aly[NCART_MAX], Alz[NCART_MAX], Blx[NCART_MAX], Bly[NCART_MAX], Blz[NCART_MAX];
    int Clx[NCART_MAX], Cly[NCART_MAX], Clz[NCART_MAX];
    fill_cart(la, Alx, Aly, Alz);
    fill_cart(lb, Blx, Bly, Blz);
    fill_cart(lc, Clx, Cly, Clz);
    double A[3], B[3], C[3];
    for (int d = 0; d < 3; ++d) {
        A[d] = ao->cxyz[3 * shA + d];
        B[d] = b_is_dummy ? 0.0 : ao->cxyz[3 * shB + d];
        C[d] = aux->cxyz[3 * shC + d];
    }
    double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double xp[3][LMAX_D + 1];
    for (int d = 0; d < 3; ++d) {
        xp[d][0] = 1.0;
        for (int k = 1; k <= LMAX_D; ++k) xp[d][k] = xp[d][k - 1] * AB[d];
    }
    int nprimA = ao->nprim[shA], nprimB = b_is_dummy ? 1 : ao->nprim[shB], nprimC = aux->nprim[shC];
    int nmax = la + lb, mmax = lc;
    int nroots = (la + lb + lc) / 2 + 1;
    double roots[NROOTS_MAX], weights[NROOTS_MAX];
    double Gx[STRIDE * STRIDE], Gy[STRIDE * STRIDE], Gz[STRIDE * STRIDE];
    memset(out, 0, sizeof(double) * nA * nB * nC);
    for (int ipA = 0; ipA < nprimA; ++ipA) {
        double a = ao->pexp[ao->pstart[shA] + ipA], ca = ao->pcoef[ao->pstart[shA] + ipA];
        for (int ipB = 0; ipB < nprimB; ++ipB) {
            double b = b_is_dummy ? 0.0 : ao->pexp[ao->pstart[shB] + ipB];
            double cb = b_is_dummy ? 1.0 : ao->pcoef[ao->pstart[shB] + ipB];
            double p = a + b, inv_p = 1.0 / p, mu = a * b * inv_p;
            double P[3];
            for (int d = 0; d < 3; ++d) P[d] = (a * A[d] + b * B[d]) * inv_p;
            double cKab = (ca * cb) * exp(-mu * AB2);
            for (int ipC = 0; ipC < nprimC; ++ipC) {
                double q = aux->pexp[aux->pstart[shC] + ipC];
                double cKcd = aux->pcoef[aux->pstart[shC] + ipC];
                double denom = p + q, inv_denom = 1.0 / denom;
                double PQ2 = 0.0;
                for (int d = 0; d < 3; ++d) PQ2 += (P[d] - C[d]) * (P[d] - C[d]);
                double T = p * q * inv_denom * PQ2;
                double base = kTwoPi52 / (p * q * sqrt(denom)) * cKab * cKcd;
                oracle_rys_roots(nroots, T, roots, weights);
                for (int u = 0; u < nroots; ++u) {
                    double x = roots[u], w = weights[u];
                    double B0 = x * 0.5 * inv_denom;
                    double B1 = (1.0 - x) * 0.5 / p + B0;
                    double B1p = (1.0 - x) * 0.5 / q + B0;
                    double Cc[3], Cp[3];
                    for (int d = 0; d < 3; ++d) {
                        Cc[d] = (P[d] - A[d]) + (q * inv_denom) * x * (C[d] - P[d]);
                        Cp[d] = (C[d] - C[d]) + (p * inv_denom) * x * (P[d] - C[d]);
                    }
                    compute_G(Gx, nmax, mmax, Cc[0], Cp[0], B0, B1, B1p);
                    compute_G(Gy, nmax, mmax, Cc[1], Cp[1], B0, B1, B1p);
                    compute_G(Gz, nmax, mmax, Cc[2], Cp[2], B0, B1, B1p);
                    double scale = base * w;
                    for (int ia = 0; ia < nA; ++ia)
                        for (int ib = 0; ib < nB; ++ib)
                            for (int ic = 0; ic < nC; ++ic) {
                                double Ix = shift_ld0(Gx, Alx[ia], Blx[ib], Clx[ic], xp[0]);
                                double Iy = shift_ld0(Gy, Aly[ia], Bly[ib], Cly[ic], xp[1]);
                                double Iz = shift_ld0(Gz, Alz[ia], Blz[ib], Clz[ic], xp[2]);
                                out[(ia * nB + ib) * nC + ic] += scale * (Ix * Iy * Iz);
                            }
                }
            }
        }
    }
}

/* ---- derivative contraction: sum_{abc} bar[abc] * d(ab|c)/dR for centres A, B, C ---- */
static void deriv_3c(const basis_t *ao, int shA, int shB, int b_is_dummy, const basis_t *aux, int shC,
                     const double *bar, double *g /* [3][3]: A, B, C x (x,y,z) */) {
    int la = ao->l[shA], lb = b_is_dummy ? 0 : ao->l[shB], lc = aux->l[shC];
    int nA = ncart(la), nB = ncart(lb), nC = ncart(lc);
    int Al[3][NCART_MAX], Bl[3][NCART_MAX], Cl[3][NCART_MAX];
    fill_cart(la, Al[0], Al[1], Al[2]);
    fill_cart(lb, Bl[0], Bl[1], Bl[2]);
    fill_cart(lc, Cl[0], Cl[1], Cl[2]);
    double A[3], B[3], C[3];
    for (int d = 0; d < 3; ++d) {
        A[d] = ao->cxyz[3 * shA + d];
        B[d] = b_is_dummy ? 0.0 : ao->cxyz[3 * shB + d];
        C[d] = aux->cxyz[3 * shC + d];
    }
    double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double xp[3][LMAX_D + 2];
    for (int d = 0; d < 3; ++d) {
        xp[d][0] = 1.0;
        for (int k = 1; k <= LMAX_D + 1; ++k) xp[d][k] = xp[d][k - 1] * AB[d];
    }
    int nprimA = ao->nprim[shA], nprimB = b_is_dummy ? 1 : ao->nprim[shB], nprimC = aux->nprim[shC];
    int nmax = la + lb + 1, mmax = lc + 1;
    int nroots = (la + lb + lc + 1) / 2 + 1;
    double roots[NROOTS_MAX], weights[NROOTS_MAX];
    double G[3][STRIDE * STRIDE];
    for (int k = 0; k < 9; ++k) g[k] = 0.0;
    for (int ipA = 0; ipA < nprimA; ++ipA) {
        double a = ao->pexp[ao->pstart[shA] + ipA], ca = ao->pcoef[ao->pstart[shA] + ipA];
        for (int ipB = 0; ipB < nprimB; ++ipB) {
            double b = b_is_dummy ? 0.0 : ao->pexp[ao->pstart[shB] + ipB];
            double cb = b_is_dummy ? 1.0 : ao->pcoef[ao->pstart[shB] + ipB];
            double p = a + b, inv_p = 1.0 / p, mu = a * b * inv_p;
            double P[3];
            for (int d = 0; d < 3; ++d) P[d] = (a * A[d] + b * B[d]) * inv_p;
            double cKab = (ca * cb) * exp(-mu * AB2);
            for (int ipC = 0; ipC < nprimC; ++ipC) {
                double q = aux->pexp[aux->pstart[shC] + ipC];
                double cKcd = aux->pcoef[aux->pstart[shC] + ipC];
                double cexp = q;
                double denom = p + q, inv_denom = 1.0 / denom;
                double PQ2 = 0.0;
                for (int d = 0; d < 3; ++d) PQ2 += (P[d] - C[d]) * (P[d] - C[d]);
                double T = p * q * inv_denom * PQ2;
                double base = kTwoPi52 / (p * q * sqrt(denom)) * cKab * cKcd;
                oracle_rys_roots(nroots, T, roots, weights);
                for (int u = 0; u < nroots; ++u) {
                    double x = roots[u], w = weights[u];
                    double B0 = x * 0.5 * inv_denom;
                    double B1 = (1.0 - x) * 0.5 / p + B0;
                    double B1p = (1.0 - x) * 0.5 / q + B0;
                    for (int d = 0; d < 3; ++d) {
                        double Cc = (P[d] - A[d]) + (q * inv_denom) * x * (C[d] - P[d]);
                        double Cp = (p * inv_denom) * x * (P[d] - C[d]);
                        compute_G(G[d], nmax, mmax, Cc, Cp, B0, B1, B1p);
                    }
                    double scale = base * w;
                    for (int ia = 0; ia < nA; ++ia)
                        for (int ib = 0; ib < nB; ++ib)
                            for (int ic = 0; ic < nC; ++ic) {
                                double bv = bar[(ia * nB + ib) * nC + ic];
                                if (bv == 0.0) continue;
                                double I[3], dA[3], dB[3], dC[3];
                                for (int d = 0; d < 3; ++d) {
                                    int i = Al[d][ia], j = Bl[d][ib], k = Cl[d][ic];
                                    I[d] = shift_ld0(G[d], i, j, k, xp[d]);
                                    double m = i > 0 ? shift_ld0(G[d], i - 1, j, k, xp[d]) : 0.0;
                                    dA[d] = -(double)i * m + 2.0 * a * shift_ld0(G[d], i + 1, j, k, xp[d]);
                                    m = j > 0 ? shift_ld0(G[d], i, j - 1, k, xp[d]) : 0.0;
                                    dB[d] = -(double)j * m + 2.0 * b * shift_ld0(G[d], i, j + 1, k, xp[d]);
                                    m = k > 0 ? shift_ld0(G[d], i, j, k - 1, xp[d]) : 0.0;
                                    dC[d] = -(double)k * m + 2.0 * cexp * shift_ld0(G[d], i, j, k + 1, xp[d]);
                                }
                                double s = bv * scale;
                                g[0] += s * dA[0] * I[1] * I[2];
                                g[1] += s * I[0] * dA[1] * I[2];
                                g[2] += s * I[0] * I[1] * dA[2];
                                g[3] += s * dB[0] * I[1] * I[2];
                                g[4] += s * I[0] * dB[1] * I[2];
                                g[5] += s * I[0] * I[1] * dB[2];
                                g[6] += s * dC[0] * I[1] * I[2];
                                g[7] += s * I[0] * dC[1] * I[2];
                                g[8] += s * I[0] * I[1] * dC[2];
                            }
                }
            }
        }
    }
}

/* ===================== exported entry points ===================== */

static basis_t mk(const double *cxyz, const int *l, const int *ps, const int *np, const double *e, const double *c) {
    basis_t b = {cxyz, l, ps, np, e, c};
    return b;
}

/* One 3c tile (A B | C); out[(ia*nB+ib)*nC+ic]. */
void oracle_tile_3c(const double *ao_cxyz, const int *ao_l, const int *ao_ps, const int *ao_np, const double *ao_e,
                    const double *ao_c, const double *ax_cxyz, const int *ax_l, const int *ax_ps, const int *ax_np,
                    const double *ax_e, const double *ax_c, int shA, int shB, int shC, double *out) {
    basis_t ao = mk(ao_cxyz, ao_l, ao_ps, ao_np, ao_e, ao_c), ax = mk(ax_cxyz, ax_l, ax_ps, ax_np, ax_e, ax_c);
    tile_3c(&ao, shA, shB, 0, &ax, shC, out);
}

/* One metric tile (P | Q); out[iP*nQ+iQ]. Both shells from the aux basis. */
void oracle_tile_2c(const double *ax_cxyz, const int *ax_l, const int *ax_ps, const int *ax_np, const double *ax_e,
                    const double *ax_c, int shP, int shQ, double *out) {
    basis_t ax = mk(ax_cxyz, ax_l, ax_ps, ax_np, ax_e, ax_c);
    tile_3c(&ax, shP, 0, 1, &ax, shQ, out);
}

/* Full X[mu, nu, P] = (mu nu | P) (nao*nao*naux), both (mu,nu) orders written. */
void oracle_int3c_full(const double *ao_cxyz, const int *ao_l, const int *ao_ps, const int *ao_np, const double *ao_e,
                       const double *ao_c, const int *ao_start, int nsh_ao, int nao, const double *ax_cxyz,
                       const int *ax_l, const int *ax_ps, const int *ax_np, const double *ax_e, const double *ax_c,
                       const int *ax_start, int nsh_ax, int naux, const int *sp_A, const int *sp_B, int nsp,
                       double *X) {
    basis_t ao = mk(ao_cxyz, ao_l, ao_ps, ao_np, ao_e, ao_c), ax = mk(ax_cxyz, ax_l, ax_ps, ax_np, ax_e, ax_c);
    (void)nsh_ao;
#pragma omp parallel for schedule(dynamic, 1)
    for (int sp = 0; sp < nsp; ++sp) {
        int A = sp_A[sp], B = sp_B[sp];
        int nA = ncart(ao_l[A]), nB = ncart(ao_l[B]);
        double *tile = (double *)malloc(sizeof(double) * nA * nB * NCART_MAX);
        for (int C = 0; C < nsh_ax; ++C) {
            int nC = ncart(ax_l[C]);
            tile_3c(&ao, A, B, 0, &ax, C, tile);
            for (int ia = 0; ia < nA; ++ia)
                for (int ib = 0; ib < nB; ++ib)
                    for (int ic = 0; ic < nC; ++ic) {
                        double v = tile[(ia * nB + ib) * nC + ic];
                        long mu = ao_start[A] + ia, nu = ao_start[B] + ib, P = ax_start[C] + ic;
                        X[(mu * nao + nu) * naux + P] = v;
                        X[(nu * nao + mu) * naux + P] = v;
                    }
        }
        free(tile);
    }
}

/* Full metric V[P, Q] (naux*naux), symmetric. */
void oracle_metric_full(const double *ax_cxyz, const int *ax_l, const int *ax_ps, const int *ax_np,
                        const double *ax_e, const double *ax_c, const int *ax_start, int nsh_ax, int naux,
                        double *V) {
    basis_t ax = mk(ax_cxyz, ax_l, ax_ps, ax_np, ax_e, ax_c);
#pragma omp parallel for schedule(dynamic, 1)
    for (int P = 0; P < nsh_ax; ++P) {
        double tile[NCART_MAX * NCART_MAX];
        int nP = ncart(ax_l[P]);
        for (int Q = 0; Q <= P; ++Q) {
            int nQ = ncart(ax_l[Q]);
            tile_3c(&ax, P, 0, 1, &ax, Q, tile);
            for (int i = 0; i < nP; ++i)
                for (int j = 0; j < nQ; ++j) {
                    long p = ax_start[P] + i, q = ax_start[Q] + j;
                    V[p * naux + q] = tile[i * nQ + j];
                    V[q * naux + p] = tile[i * nQ + j];
                }
        }
    }
}

/*
 * 3c gradient contraction (asuka/integrals/grad.py:420-458): for every AO
 * shell pair (A>=B, l-ordered) and aux shell C,
 *   grad[atom(A)] += fac * sum bar * d/dA,  same for B and C,  fac = 2 if A != B.
 * bar_X is (nao, nao, naux), symmetric in (mu, nu).  grad is (natm, 3), accumulated.
 */
void oracle_deriv3c_full(const double *ao_cxyz, const int *ao_l, const int *ao_ps, const int *ao_np,
                         const double *ao_e, const double *ao_c, const int *ao_start, const int *ao_atom, int nao,
                         const double *ax_cxyz, const int *ax_l, const int *ax_ps, const int *ax_np,
                         const double *ax_e, const double *ax_c, const int *ax_start, const int *ax_atom, int nsh_ax,
                         int naux, const int *sp_A, const int *sp_B, int nsp, const double *barX, int natm,
                         double *grad) {
    basis_t ao = mk(ao_cxyz, ao_l, ao_ps, ao_np, ao_e, ao_c), ax = mk(ax_cxyz, ax_l, ax_ps, ax_np, ax_e, ax_c);
    double *acc = (double *)calloc((size_t)natm * 3, sizeof(double));
#pragma omp parallel
    {
        double *loc = (double *)calloc((size_t)natm * 3, sizeof(double));
        double *bar = (double *)malloc(sizeof(double) * NCART_MAX * NCART_MAX * NCART_MAX);
#pragma omp for schedule(dynamic, 1)
        for (int sp = 0; sp < nsp; ++sp) {
            int A = sp_A[sp], B = sp_B[sp];
            int nA = ncart(ao_l[A]), nB = ncart(ao_l[B]);
            double fac = (A != B) ? 2.0 : 1.0;
            for (int C = 0; C < nsh_ax; ++C) {
                int nC = ncart(ax_l[C]);
                for (int ia = 0; ia < nA; ++ia)
                    for (int ib = 0; ib < nB; ++ib)
                        for (int ic = 0; ic < nC; ++ic) {
                            long mu = ao_start[A] + ia, nu = ao_start[B] + ib, P = ax_start[C] + ic;
                            bar[(ia * nB + ib) * nC + ic] = barX[(mu * nao + nu) * naux + P];
                        }
                double g[9];
                deriv_3c(&ao, A, B, 0, &ax, C, bar, g);
                for (int d = 0; d < 3; ++d) {
                    loc[3 * ao_atom[A] + d] += fac * g[d];
                    loc[3 * ao_atom[B] + d] += fac * g[3 + d];
                    loc[3 * ax_atom[C] + d] += fac * g[6 + d];
                }
            }
        }
#pragma omp critical
        for (int k = 0; k < natm * 3; ++k) acc[k] += loc[k];
        free(loc);
        free(bar);
    }
    for (int k = 0; k < natm * 3; ++k) grad[k] += acc[k];
    free(acc);
}

/*
 * 2c gradient contraction (asuka/integrals/grad.py:573-616): for P >= Q,
 * grad[atom(P)] += fac * sum bar_V d/dP, grad[atom(Q)] += fac * sum bar_V d/dQ,
 * fac = 2 if P != Q.  bar_V is (naux, naux) symmetric.
 */
void oracle_deriv2c_full(const double *ax_cxyz, const int *ax_l, const int *ax_ps, const int *ax_np,
                         const double *ax_e, const double *ax_c, const int *ax_start, const int *ax_atom, int nsh_ax,
                         int naux, const double *barV, int natm, double *grad) {
    basis_t ax = mk(ax_cxyz, ax_l, ax_ps, ax_np, ax_e, ax_c);
    double *acc = (double *)calloc((size_t)natm * 3, sizeof(double));
#pragma omp parallel
    {
        double *loc = (double *)calloc((size_t)natm * 3, sizeof(double));
        double bar[NCART_MAX * NCART_MAX];
#pragma omp for schedule(dynamic, 1)
        for (int P = 0; P < nsh_ax; ++P) {
            int nP = ncart(ax_l[P]);
            for (int Q = 0; Q <= P; ++Q) {
                int nQ = ncart(ax_l[Q]);
                double fac = (P != Q) ? 2.0 : 1.0;
                for (int i = 0; i < nP; ++i)
                    for (int j = 0; j < nQ; ++j) bar[i * nQ + j] = barV[(long)(ax_start[P] + i) * naux + ax_start[Q] + j];
                double g[9];
                deriv_3c(&ax, P, 0, 1, &ax, Q, bar, g);
                for (int d = 0; d < 3; ++d) {
                    loc[3 * ax_atom[P] + d] += fac * g[d];
                    loc[3 * ax_atom[Q] + d] += fac * g[6 + d];
                }
            }
        }
#pragma omp critical
        for (int k = 0; k < natm * 3; ++k) acc[k] += loc[k];
        free(loc);
    }
    for (int k = 0; k < natm * 3; ++k) grad[k] += acc[k];
    free(acc);
}
