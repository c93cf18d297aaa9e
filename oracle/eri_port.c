/*
 * ORACLE - test infrastructure only (see eri_port.h).  A direct, unoptimised restatement in C of
 * the reference's electron-repulsion integrals (MihkuU/Lible, src/lible/ints), written for clarity:
 *
 *   Boys function          src/lible/ints/boys_function.cpp:6-118 (grid step 0.01 on [0,30],
 *                          7-term Taylor + downward recursion, asymptotic beyond 30)
 *   Hermite E recurrences   src/lible/ints/ecoeffs.cpp:33-111 (E and dE/d(A-B))
 *   spherical transform     src/lible/ints/spherical_trafo.cpp (real solid harmonics, m = 0,+1,-1,...)
 *   AO norms                src/lible/ints/shell.cpp:11-46 (spherical self-overlap)
 *   pair screening / order  src/lible/ints/shell_pair_data.cpp:73-202
 *   SHARK E matrices        src/lible/ints/ecoeffs.cpp:314-517
 *   R recursion             src/lible/ints/rints.hpp:112-213
 *   quartet                 src/lible/ints/twoel/eri_kernel_funs.hpp:104-193 (and D1: 350-515)
 *   eri4 driver             src/lible/ints/twoel/eri4.cpp:38-95
 * J/K digestion and the J/K energy gradient have no reference implementation; they follow the
 * same unique-quartet enumeration and 8-fold symmetry weights as the engine's restatement on the
 * reference kernels (oracle/ref_capi.cpp).
 */
#define _GNU_SOURCE
#include "eri_port.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXL 5
#define MAXLT 16
#define BOYS_ROWS 3001
#define BOYS_COLS 24

static double g_boys[BOYS_ROWS * BOYS_COLS];
static int g_boys_ready = 0;

static int nherm(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }
static int nsph(int l) { return 2 * l + 1; }
static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int herm_index(int t, int u, int v)
{
    int jk = u + v;
    return nherm(t + u + v - 1) + jk * (jk + 1) / 2 + v;
}

/* ---- Boys function ------------------------------------------------------------------------ */
static void boys_init(void)
{
    if (g_boys_ready)
        return;
    const int nmax = BOYS_COLS - 1;
    for (int k = 0; k < BOYS_ROWS; k++)
    {
        double x = k * 0.01;
        double term = 1.0 / (2.0 * nmax + 1.0), sum = term;
        for (int i = 1;; i++)
        {
            term *= x / (nmax + 0.5 + i);
            sum += term;
            if (fabs(term) < 1e-16)
                break;
        }
        double ex = exp(-x);
        double *row = g_boys + (size_t)k * BOYS_COLS;
        row[nmax] = ex * sum;
        for (int n = nmax - 1; n >= 0; n--)
            row[n] = (2.0 * x * row[n + 1] + ex) / (2 * n + 1);
    }
    g_boys_ready = 1;
}

void port_boys(int n, double x, double *F)
{
    boys_init();
    if (x == 0.0)
    {
        F[0] = 1.0;
        for (int k = 1; k <= n; k++)
            F[k] = 1.0 / (2 * k + 1);
    }
    else if (x > 30.0)
    {
        F[0] = 0.5 * sqrt(M_PI / x);
        for (int k = 1; k <= n; k++)
            F[k] = F[k - 1] * (k - 0.5) / x;
    }
    else
    {
        int iv = (int)(x / 0.01);
        double dx = x - iv * 0.01, pk = 1.0, fact = 1.0;
        const double *row = g_boys + (size_t)iv * BOYS_COLS;
        double s = row[n];
        for (int k = 1; k < 7; k++)
        {
            pk *= -dx;
            fact *= k;
            s += row[n + k] * pk / fact;
        }
        F[n] = s;
        double ex = exp(-x);
        for (int k = n - 1; k >= 0; k--)
            F[k] = (2.0 * x * F[k + 1] + ex) / (2 * k + 1);
    }
}

/* ---- Hermite E coefficients along one axis: E[i][j][t] ----------------------------------- */
#define EIDX(i, j, t) (((i) * (lb + 1) + (j)) * (la + lb + 1) + (t))
static void ecoef(int la, int lb, double a, double b, double pa, double pb, double kab, double *E)
{
    const double o2p = 1.0 / (2.0 * (a + b));
    memset(E, 0, sizeof(double) * (la + 1) * (lb + 1) * (la + lb + 1));
    E[EIDX(0, 0, 0)] = kab;
    for (int i = 1; i <= la; i++)
        for (int t = 0; t <= i; t++)
            E[EIDX(i, 0, t)] = pa * E[EIDX(i - 1, 0, t)] + (t > 0 ? o2p * E[EIDX(i - 1, 0, t - 1)] : 0.0) +
                               (t + 1 <= i - 1 ? (t + 1) * E[EIDX(i - 1, 0, t + 1)] : 0.0);
    for (int j = 1; j <= lb; j++)
        for (int i = 0; i <= la; i++)
            for (int t = 0; t <= i + j; t++)
                E[EIDX(i, j, t)] = pb * E[EIDX(i, j - 1, t)] + (t > 0 ? o2p * E[EIDX(i, j - 1, t - 1)] : 0.0) +
                                   (t + 1 <= i + j - 1 ? (t + 1) * E[EIDX(i, j - 1, t + 1)] : 0.0);
}

/* dE/dR with R = A - B (src/lible/ints/ecoeffs.cpp:70-111) */
static void ecoef1(int la, int lb, double a, double b, double r, const double *E, double *E1)
{
    const double p = a + b, o2p = 1.0 / (2.0 * p), pa = -(b / p) * r, pb = (a / p) * r;
    memset(E1, 0, sizeof(double) * (la + 1) * (lb + 1) * (la + lb + 1));
    E1[EIDX(0, 0, 0)] = -2.0 * a * b / p * r * E[EIDX(0, 0, 0)];
    for (int i = 1; i <= la; i++)
        for (int t = 0; t <= i; t++)
            E1[EIDX(i, 0, t)] = pa * E1[EIDX(i - 1, 0, t)] - (b / p) * E[EIDX(i - 1, 0, t)] +
                                (t > 0 ? o2p * E1[EIDX(i - 1, 0, t - 1)] : 0.0) +
                                (t + 1 <= i - 1 ? (t + 1) * E1[EIDX(i - 1, 0, t + 1)] : 0.0);
    for (int j = 1; j <= lb; j++)
        for (int i = 0; i <= la; i++)
            for (int t = 0; t <= i + j; t++)
                E1[EIDX(i, j, t)] = pb * E1[EIDX(i, j - 1, t)] + (a / p) * E[EIDX(i, j - 1, t)] +
                                    (t > 0 ? o2p * E1[EIDX(i, j - 1, t - 1)] : 0.0) +
                                    (t + 1 <= i + j - 1 ? (t + 1) * E1[EIDX(i, j - 1, t + 1)] : 0.0);
}

/* ---- spherical transformation: T[row][cart] (dense), HJO eqs. 6.4.47-6.4.50 --------------- */
static double binom(int n, int k)
{
    if (k < 0 || k > n)
        return 0.0;
    double r = 1.0;
    for (int i = 1; i <= k; i++)
        r = r * (n - k + i) / i;
    return r;
}

static double fact(int n)
{
    double r = 1.0;
    for (int i = 2; i <= n; i++)
        r *= i;
    return r;
}

static void sph_trafo(int l, double *T /* [2l+1][ncart] */)
{
    int nc = ncart(l);
    memset(T, 0, sizeof(double) * nsph(l) * nc);
    for (int row = 0; row < nsph(l); row++)
    {
        int m = row == 0 ? 0 : (row % 2 ? (row + 1) / 2 : -(row / 2));
        int am = abs(m);
        double N = sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0)) / (pow(2.0, am) * fact(l));
        for (int t = 0; t <= (l - am) / 2; t++)
            for (int u = 0; u <= t; u++)
                for (int tv = (m < 0 ? 1 : 0); tv <= am; tv += 2)
                {
                    int se = t + (m < 0 ? (tv - 1) / 2 : tv / 2);
                    double c = (se % 2 ? -1.0 : 1.0) * pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                               binom(t, u) * binom(am, tv);
                    int py = 2 * u + tv, px = 2 * t + am - 2 * u - tv, pz = l - 2 * t - am;
                    if (px < 0 || py < 0 || pz < 0)
                        continue;
                    int jk = py + pz;
                    T[row * nc + jk * (jk + 1) / 2 + pz] += N * c;
                }
    }
}

static void cart_exps(int l, int c, int *x, int *y, int *z)
{
    for (int i = l, k = 0; i >= 0; i--)
        for (int j = l - i; j >= 0; j--, k++)
            if (k == c)
            {
                *x = i;
                *y = j;
                *z = l - i - j;
            }
}

/* ---- molecule ------------------------------------------------------------------------------- */
typedef struct
{
    int l, atom, ao, idx, np;
    double xyz[3];
    double *e, *d; /* exponents, coefficients incl. primitive norms */
    double norm[2 * MAXL + 1];
} pshell;

typedef struct
{
    int la, lb, n, nprim;
    int *sa, *sb, *pofs, *ia, *ib;
    double *ea, *eb, *E, *E1, *P, *Q;
} pclass;

struct port_mol
{
    int nat, nsh, nao, lmax, ncls;
    double *xyz;
    pshell *sh;
    pclass *cls;
};

static double prim_norm(int l, double a)
{
    double df = 1.0;
    for (int i = 2 * l - 1; i >= 2; i -= 2)
        df *= i;
    return sqrt(pow(2 * a / M_PI, 1.5) * pow(4 * a, l) / df);
}

static void shell_norms(pshell *s)
{
    int l = s->l, nc = ncart(l), ns = nsph(l);
    double *S = calloc(nc * nc, sizeof(double)), *T = malloc(sizeof(double) * ns * nc);
    double E[(MAXL + 1) * (MAXL + 1) * (2 * MAXL + 1)];
    for (int i = 0; i < s->np; i++)
        for (int j = 0; j < s->np; j++)
        {
            double p = s->e[i] + s->e[j];
            double f = s->d[i] * s->d[j] * pow(M_PI / p, 1.5);
            int la = l, lb = l;
            ecoef(l, l, s->e[i], s->e[j], 0.0, 0.0, 1.0, E);
            for (int m = 0; m < nc; m++)
                for (int n = 0; n < nc; n++)
                {
                    int mx, my, mz, nx, ny, nz;
                    cart_exps(l, m, &mx, &my, &mz);
                    cart_exps(l, n, &nx, &ny, &nz);
                    S[m * nc + n] += f * E[EIDX(mx, nx, 0)] * E[EIDX(my, ny, 0)] * E[EIDX(mz, nz, 0)];
                }
            (void)la;
            (void)lb;
        }
    sph_trafo(l, T);
    for (int r = 0; r < ns; r++)
    {
        double v = 0.0;
        for (int m = 0; m < nc; m++)
            for (int n = 0; n < nc; n++)
                v += T[r * nc + m] * T[r * nc + n] * S[m * nc + n];
        s->norm[r] = 1.0 / sqrt(v);
    }
    free(S);
    free(T);
}

/* SHARK E (and dE/d(A-B)) for every primitive pair of a class */
static void class_ecoeffs(pclass *c, const pshell *sh)
{
    int la = c->la, lb = c->lb, sa = nsph(la), sb = nsph(lb), hab = nherm(la + lb);
    int nca = ncart(la), ncb = ncart(lb);
    double *Ta = malloc(sizeof(double) * sa * nca), *Tb = malloc(sizeof(double) * sb * ncb);
    sph_trafo(la, Ta);
    sph_trafo(lb, Tb);
    c->E = calloc((size_t)c->nprim * sa * sb * hab, sizeof(double));
    c->E1 = calloc((size_t)c->nprim * 3 * sa * sb * hab, sizeof(double));
    c->P = malloc(sizeof(double) * 3 * c->nprim);
    double Ex[3][(MAXL + 1) * (MAXL + 1) * (2 * MAXL + 1)], E1x[3][(MAXL + 1) * (MAXL + 1) * (2 * MAXL + 1)];
    for (int ip = 0; ip < c->n; ip++)
    {
        const pshell *A = &sh[c->sa[ip]], *B = &sh[c->sb[ip]];
        for (int k = c->pofs[ip]; k < c->pofs[ip + 1]; k++)
        {
            double a = c->ea[k], b = c->eb[k], p = a + b, mu = a * b / p;
            double dd = A->d[c->ia[k]] * B->d[c->ib[k]];
            for (int x = 0; x < 3; x++)
            {
                double P = (a * A->xyz[x] + b * B->xyz[x]) / p;
                c->P[3 * k + x] = P;
                double r = A->xyz[x] - B->xyz[x];
                ecoef(la, lb, a, b, P - A->xyz[x], P - B->xyz[x], exp(-mu * r * r), Ex[x]);
                ecoef1(la, lb, a, b, r, Ex[x], E1x[x]);
            }
            for (int m = 0; m < sa; m++)
                for (int n = 0; n < sb; n++)
                {
                    double s = A->norm[m] * B->norm[n] * dd;
                    double *e0 = c->E + ((size_t)k * sa * sb + m * sb + n) * hab;
                    for (int ca = 0; ca < nca; ca++)
                    {
                        if (Ta[m * nca + ca] == 0.0)
                            continue;
                        int ax, ay, az;
                        cart_exps(la, ca, &ax, &ay, &az);
                        for (int cb = 0; cb < ncb; cb++)
                        {
                            if (Tb[n * ncb + cb] == 0.0)
                                continue;
                            int bx, by, bz;
                            cart_exps(lb, cb, &bx, &by, &bz);
                            double w = s * Ta[m * nca + ca] * Tb[n * ncb + cb];
                            for (int t = 0; t <= ax + bx; t++)
                                for (int u = 0; u <= ay + by; u++)
                                    for (int v = 0; v <= az + bz; v++)
                                    {
                                        int h = herm_index(t, u, v);
                                        double gx = Ex[0][EIDX(ax, bx, t)], gy = Ex[1][EIDX(ay, by, u)],
                                               gz = Ex[2][EIDX(az, bz, v)];
                                        e0[h] += w * gx * gy * gz;
                                        double *e1 = c->E1 + (((size_t)k * 3) * sa * sb + m * sb + n) * hab;
                                        size_t st = (size_t)sa * sb * hab;
                                        e1[h] += w * E1x[0][EIDX(ax, bx, t)] * gy * gz;
                                        e1[st + h] += w * gx * E1x[1][EIDX(ay, by, u)] * gz;
                                        e1[2 * st + h] += w * gx * gy * E1x[2][EIDX(az, bz, v)];
                                    }
                        }
                    }
                }
        }
    }
    free(Ta);
    free(Tb);
}

port_mol *port_new(int n_atoms, const int *Z, const double *xyz, const int *nsh, const int *sl, const int *snp,
                   const double *exps, const double *coeffs)
{
    (void)Z;
    boys_init();
    port_mol *m = calloc(1, sizeof(port_mol));
    m->nat = n_atoms;
    m->xyz = malloc(sizeof(double) * 3 * n_atoms);
    memcpy(m->xyz, xyz, sizeof(double) * 3 * n_atoms);
    int total = 0;
    for (int a = 0; a < n_atoms; a++)
        total += nsh[a];
    m->nsh = total;
    m->sh = calloc(total, sizeof(pshell));
    int is = 0, ip = 0, ao = 0;
    for (int a = 0; a < n_atoms; a++)
        for (int k = 0; k < nsh[a]; k++, is++)
        {
            pshell *s = &m->sh[is];
            s->l = sl[is];
            s->atom = a;
            s->ao = ao;
            s->idx = is;
            s->np = snp[is];
            memcpy(s->xyz, xyz + 3 * a, sizeof(double) * 3);
            s->e = malloc(sizeof(double) * s->np);
            s->d = malloc(sizeof(double) * s->np);
            for (int p = 0; p < s->np; p++, ip++)
            {
                s->e[p] = exps[ip];
                s->d[p] = coeffs[ip] * prim_norm(s->l, exps[ip]);
            }
            shell_norms(s);
            ao += nsph(s->l);
            if (s->l > m->lmax)
                m->lmax = s->l;
        }
    m->nao = ao;
    m->ncls = (m->lmax + 1) * (m->lmax + 2) / 2;
    m->cls = calloc(m->ncls, sizeof(pclass));
    int ic = 0;
    for (int la = 0; la <= m->lmax; la++)
        for (int lb = 0; lb <= la; lb++, ic++)
        {
            pclass *c = &m->cls[ic];
            c->la = la;
            c->lb = lb;
            int cap = total * total + 1, tp = 0;
            for (int i = 0; i < total; i++)
                tp += m->sh[i].np;
            size_t pcap = (size_t)tp * tp + 1;
            c->sa = malloc(sizeof(int) * cap);
            c->sb = malloc(sizeof(int) * cap);
            c->pofs = malloc(sizeof(int) * (cap + 1));
            c->ea = malloc(sizeof(double) * pcap);
            c->eb = malloc(sizeof(double) * pcap);
            c->ia = malloc(sizeof(int) * pcap);
            c->ib = malloc(sizeof(int) * pcap);
            c->pofs[0] = 0;
            int np = 0;
            for (int i = 0; i < total; i++)
            {
                if (m->sh[i].l != la)
                    continue;
                for (int j = 0; j < total; j++)
                {
                    if (m->sh[j].l != lb)
                        continue;
                    if (la == lb && j > i)
                        break;
                    const pshell *A = &m->sh[i], *B = &m->sh[j];
                    double r2 = 0;
                    for (int x = 0; x < 3; x++)
                        r2 += (A->xyz[x] - B->xyz[x]) * (A->xyz[x] - B->xyz[x]);
                    int kept = 0;
                    for (int p = 0; p < A->np; p++)
                        for (int q = 0; q < B->np; q++)
                        {
                            double a = A->e[p], b = B->e[q];
                            if (fabs(A->d[p] * B->d[q] * exp(-a * b / (a + b) * r2)) >= 1e-15)
                            {
                                c->ea[np] = a;
                                c->eb[np] = b;
                                c->ia[np] = p;
                                c->ib[np] = q;
                                np++;
                                kept++;
                            }
                        }
                    if (!kept)
                        continue;
                    c->sa[c->n] = i;
                    c->sb[c->n] = j;
                    c->n++;
                    c->pofs[c->n] = np;
                }
            }
            c->nprim = np;
            class_ecoeffs(c, m->sh);
        }
    return m;
}

void port_free(port_mol *m)
{
    if (!m)
        return;
    for (int i = 0; i < m->nsh; i++)
    {
        free(m->sh[i].e);
        free(m->sh[i].d);
    }
    for (int c = 0; c < m->ncls; c++)
    {
        pclass *x = &m->cls[c];
        free(x->sa);
        free(x->sb);
        free(x->pofs);
        free(x->ea);
        free(x->eb);
        free(x->ia);
        free(x->ib);
        free(x->E);
        free(x->E1);
        free(x->P);
        free(x->Q);
    }
    free(m->cls);
    free(m->sh);
    free(m->xyz);
    free(m);
}

int port_nao(const port_mol *m) { return m->nao; }

/* ---- R integrals: R[h] for t+u+v <= L at n = 0 (src/lible/ints/rints.hpp:112-175) ---------- */
static void rints(int L, double alpha, const double *F, double X, double Y, double Z, double *R, double *buf)
{
    /* buf: (L+1) levels x nherm(L) */
    int nh = nherm(L);
    for (int n = L; n >= 0; n--)
    {
        double *cur = buf + (size_t)n * nh, *up = buf + (size_t)(n + 1) * nh;
        cur[0] = pow(-2.0 * alpha, n) * F[n];
        for (int o = 1; o <= L - n; o++)
            for (int t = o; t >= 0; t--)
                for (int u = o - t; u >= 0; u--)
                {
                    int v = o - t - u, h = herm_index(t, u, v);
                    double r;
                    if (t > 0)
                        r = X * up[herm_index(t - 1, u, v)] + (t > 1 ? (t - 1) * up[herm_index(t - 2, u, v)] : 0.0);
                    else if (u > 0)
                        r = Y * up[herm_index(t, u - 1, v)] + (u > 1 ? (u - 1) * up[herm_index(t, u - 2, v)] : 0.0);
                    else
                        r = Z * up[herm_index(t, u, v - 1)] + (v > 1 ? (v - 1) * up[herm_index(t, u, v - 2)] : 0.0);
                    cur[h] = r;
                }
    }
    memcpy(R, buf, sizeof(double) * nh);
}

typedef struct
{
    int t[1000], u[1000], v[1000];
} htab;
static htab g_ht;
static int g_ht_ready = 0;
static void htab_init(void)
{
    if (g_ht_ready)
        return;
    for (int n = 0, h = 0; n < 14; n++)
        for (int t = n; t >= 0; t--)
            for (int u = n - t; u >= 0; u--, h++)
            {
                g_ht.t[h] = t;
                g_ht.u[h] = u;
                g_ht.v[h] = n - t - u;
            }
    g_ht_ready = 1;
}

/* Contracted quartet; with d1 != NULL also the 12 derivative blocks [A,B,C,D][x,y,z]. */
static void quartet(const port_mol *m, const pclass *A, int i, const pclass *B, int j, double *out, double *d1)
{
    htab_init();
    int lab = A->la + A->lb, lcd = B->la + B->lb, L = lab + lcd + (d1 ? 1 : 0);
    int sab = nsph(A->la) * nsph(A->lb), scd = nsph(B->la) * nsph(B->lb);
    int hab = nherm(lab), hcd = nherm(lcd), nh = nherm(L);
    double F[MAXLT + 2], *R = malloc(sizeof(double) * nh), *buf = malloc(sizeof(double) * (L + 2) * nh);
    double *M = malloc(sizeof(double) * 4 * hab * hcd); /* R matrix + 3 shifted */
    memset(out, 0, sizeof(double) * sab * scd);
    if (d1)
        memset(d1, 0, sizeof(double) * 12 * sab * scd);
    for (int p = A->pofs[i]; p < A->pofs[i + 1]; p++)
        for (int q = B->pofs[j]; q < B->pofs[j + 1]; q++)
        {
            double pp = A->ea[p] + A->eb[p], qq = B->ea[q] + B->eb[q], alpha = pp * qq / (pp + qq);
            double X = A->P[3 * p] - B->P[3 * q], Y = A->P[3 * p + 1] - B->P[3 * q + 1],
                   Z = A->P[3 * p + 2] - B->P[3 * q + 2];
            port_boys(L, alpha * (X * X + Y * Y + Z * Z), F);
            double fac = 2.0 * pow(M_PI, 2.5) / (pp * qq * sqrt(pp + qq));
            rints(L, alpha, F, X, Y, Z, R, buf);
            for (int h = 0; h < hab; h++)
                for (int g = 0; g < hcd; g++)
                {
                    int t = g_ht.t[h] + g_ht.t[g], u = g_ht.u[h] + g_ht.u[g], v = g_ht.v[h] + g_ht.v[g];
                    double sg = ((g_ht.t[g] + g_ht.u[g] + g_ht.v[g]) % 2 ? -1.0 : 1.0) * fac;
                    M[h * hcd + g] = sg * R[herm_index(t, u, v)];
                    if (d1)
                    {
                        M[(1 * hab + h) * hcd + g] = sg * R[herm_index(t + 1, u, v)];
                        M[(2 * hab + h) * hcd + g] = sg * R[herm_index(t, u + 1, v)];
                        M[(3 * hab + h) * hcd + g] = sg * R[herm_index(t, u, v + 1)];
                    }
                }
            const double *ea = A->E + (size_t)p * sab * hab, *ec = B->E + (size_t)q * scd * hcd;
            for (int x = 0; x < sab; x++)
                for (int y = 0; y < scd; y++)
                {
                    double s = 0.0, sx[3] = {0, 0, 0}, sr[3] = {0, 0, 0}, sc[3] = {0, 0, 0};
                    for (int h = 0; h < hab; h++)
                        for (int g = 0; g < hcd; g++)
                        {
                            double w = ea[x * hab + h] * ec[y * hcd + g];
                            s += w * M[h * hcd + g];
                            if (d1)
                                for (int k = 0; k < 3; k++)
                                {
                                    sx[k] += w * M[((1 + k) * hab + h) * hcd + g];
                                    sr[k] += A->E1[(((size_t)p * 3 + k) * sab + x) * hab + h] * ec[y * hcd + g] *
                                             M[h * hcd + g];
                                    sc[k] += ea[x * hab + h] * B->E1[(((size_t)q * 3 + k) * scd + y) * hcd + g] *
                                             M[h * hcd + g];
                                }
                        }
                    out[x * scd + y] += s;
                    if (d1)
                    {
                        double a = A->ea[p], b = A->eb[p], c = B->ea[q];
                        for (int k = 0; k < 3; k++)
                        {
                            size_t o = (size_t)x * scd + y, blk = (size_t)sab * scd;
                            d1[(0 + k) * blk + o] += (a / pp) * sx[k] + sr[k];
                            d1[(3 + k) * blk + o] += (b / pp) * sx[k] - sr[k];
                            d1[(6 + k) * blk + o] += -(c / qq) * sx[k] + sc[k];
                        }
                    }
                }
        }
    if (d1)
    {
        size_t blk = (size_t)sab * scd;
        for (int k = 0; k < 3; k++)
            for (size_t o = 0; o < blk; o++)
                d1[(9 + k) * blk + o] = -(d1[k * blk + o] + d1[(3 + k) * blk + o] + d1[(6 + k) * blk + o]);
    }
    free(R);
    free(buf);
    free(M);
}

void port_eri4(const port_mol *m, double *out)
{
    const long n = m->nao;
    memset(out, 0, sizeof(double) * n * n * n * n);
    for (int cb = 0; cb < m->ncls; cb++)
        for (int ck = 0; ck <= cb; ck++)
        {
            const pclass *A = &m->cls[cb], *B = &m->cls[ck];
            int sa = nsph(A->la), sb = nsph(A->lb), sc = nsph(B->la), sd = nsph(B->lb);
#pragma omp parallel for schedule(dynamic)
            for (int i = 0; i < A->n; i++)
            {
                double *v = malloc(sizeof(double) * sa * sb * sc * sd);
                for (int j = 0; j < (cb == ck ? i + 1 : B->n); j++)
                {
                    quartet(m, A, i, B, j, v, NULL);
                    long oa = m->sh[A->sa[i]].ao, ob = m->sh[A->sb[i]].ao, oc = m->sh[B->sa[j]].ao,
                         od = m->sh[B->sb[j]].ao;
                    for (int x = 0; x < sa; x++)
                        for (int y = 0; y < sb; y++)
                            for (int z = 0; z < sc; z++)
                                for (int w = 0; w < sd; w++)
                                {
                                    double g = v[((x * sb + y) * sc + z) * sd + w];
                                    long a = oa + x, b = ob + y, c = oc + z, d = od + w;
                                    out[((a * n + b) * n + c) * n + d] = g;
                                    out[((a * n + b) * n + d) * n + c] = g;
                                    out[((b * n + a) * n + c) * n + d] = g;
                                    out[((b * n + a) * n + d) * n + c] = g;
                                    out[((c * n + d) * n + a) * n + b] = g;
                                    out[((c * n + d) * n + b) * n + a] = g;
                                    out[((d * n + c) * n + a) * n + b] = g;
                                    out[((d * n + c) * n + b) * n + a] = g;
                                }
                }
                free(v);
            }
        }
}

static void schwarz(const port_mol *m)
{
    for (int c = 0; c < m->ncls; c++)
    {
        pclass *A = &m->cls[c];
        if (A->Q)
            continue;
        int sab = nsph(A->la) * nsph(A->lb);
        double *Q = malloc(sizeof(double) * (A->n + 1));
#pragma omp parallel for schedule(dynamic)
        for (int i = 0; i < A->n; i++)
        {
            double *v = malloc(sizeof(double) * sab * sab), mx = 0.0;
            quartet(m, A, i, A, i, v, NULL);
            for (int e = 0; e < sab; e++)
                mx = fmax(mx, fabs(v[e * sab + e]));
            Q[i] = sqrt(mx);
            free(v);
        }
        A->Q = Q;
    }
}

static double weight(const pclass *A, int i, const pclass *B, int j, int same)
{
    double f = 1.0;
    if (A->sa[i] == A->sb[i])
        f *= 0.5;
    if (B->sa[j] == B->sb[j])
        f *= 0.5;
    if (same && i == j)
        f *= 0.5;
    return f;
}

long long port_jk(const port_mol *m, const double *D, double *J, double *K, double thr, int stride)
{
    const long n = m->nao;
    schwarz(m);
    memset(J, 0, sizeof(double) * n * n);
    memset(K, 0, sizeof(double) * n * n);
    long long nq = 0;
    if (stride < 1)
        stride = 1;
    for (int cb = 0; cb < m->ncls; cb++)
        for (int ck = 0; ck <= cb; ck++)
        {
            const pclass *A = &m->cls[cb], *B = &m->cls[ck];
            int sa = nsph(A->la), sb = nsph(A->lb), sc = nsph(B->la), sd = nsph(B->lb);
#pragma omp parallel for schedule(dynamic) reduction(+ : nq)
            for (int i = 0; i < A->n; i += stride)
            {
                double *v = malloc(sizeof(double) * sa * sb * sc * sd);
                for (int j = 0; j < (cb == ck ? i + 1 : B->n); j++)
                {
                    if (A->Q[i] * B->Q[j] < thr)
                        continue;
                    nq++;
                    quartet(m, A, i, B, j, v, NULL);
                    double f = weight(A, i, B, j, cb == ck);
                    long oa = m->sh[A->sa[i]].ao, ob = m->sh[A->sb[i]].ao, oc = m->sh[B->sa[j]].ao,
                         od = m->sh[B->sb[j]].ao;
                    for (int x = 0; x < sa; x++)
                        for (int y = 0; y < sb; y++)
                            for (int z = 0; z < sc; z++)
                                for (int w = 0; w < sd; w++)
                                {
                                    double g = f * v[((x * sb + y) * sc + z) * sd + w];
                                    long a = oa + x, b = ob + y, c = oc + z, d = od + w;
#pragma omp atomic
                                    J[a * n + b] += 2 * g * D[c * n + d];
#pragma omp atomic
                                    J[c * n + d] += 2 * g * D[a * n + b];
#pragma omp atomic
                                    K[a * n + c] += g * D[b * n + d];
#pragma omp atomic
                                    K[a * n + d] += g * D[b * n + c];
#pragma omp atomic
                                    K[b * n + c] += g * D[a * n + d];
#pragma omp atomic
                                    K[b * n + d] += g * D[a * n + c];
                                }
                }
                free(v);
            }
        }
    for (long r = 0; r < n; r++)
        for (long c = 0; c <= r; c++)
        {
            double j = J[r * n + c] + J[c * n + r], k = K[r * n + c] + K[c * n + r];
            J[r * n + c] = J[c * n + r] = j;
            K[r * n + c] = K[c * n + r] = k;
        }
    return nq;
}

void port_jk_grad(const port_mol *m, const double *D, double *grad)
{
    const long n = m->nao;
    memset(grad, 0, sizeof(double) * 3 * m->nat);
    for (int cb = 0; cb < m->ncls; cb++)
        for (int ck = 0; ck <= cb; ck++)
        {
            const pclass *A = &m->cls[cb], *B = &m->cls[ck];
            int sa = nsph(A->la), sb = nsph(A->lb), sc = nsph(B->la), sd = nsph(B->lb);
            size_t blk = (size_t)sa * sb * sc * sd;
#pragma omp parallel for schedule(dynamic)
            for (int i = 0; i < A->n; i++)
            {
                double *v = malloc(sizeof(double) * blk), *d1 = malloc(sizeof(double) * 12 * blk);
                for (int j = 0; j < (cb == ck ? i + 1 : B->n); j++)
                {
                    quartet(m, A, i, B, j, v, d1);
                    double f = weight(A, i, B, j, cb == ck);
                    long oa = m->sh[A->sa[i]].ao, ob = m->sh[A->sb[i]].ao, oc = m->sh[B->sa[j]].ao,
                         od = m->sh[B->sb[j]].ao;
                    int at[4] = {m->sh[A->sa[i]].atom, m->sh[A->sb[i]].atom, m->sh[B->sa[j]].atom,
                                 m->sh[B->sb[j]].atom};
                    double acc[12] = {0};
                    for (int x = 0; x < sa; x++)
                        for (int y = 0; y < sb; y++)
                            for (int z = 0; z < sc; z++)
                                for (int w = 0; w < sd; w++)
                                {
                                    long a = oa + x, b = ob + y, c = oc + z, d = od + w;
                                    double gam = f * (4 * D[a * n + b] * D[c * n + d] - D[a * n + c] * D[b * n + d] -
                                                      D[a * n + d] * D[b * n + c]);
                                    size_t e = ((x * sb + y) * sc + z) * sd + w;
                                    for (int k = 0; k < 12; k++)
                                        acc[k] += gam * d1[k * blk + e];
                                }
                    for (int k = 0; k < 12; k++)
                    {
#pragma omp atomic
                        grad[3 * at[k / 3] + k % 3] += acc[k];
                    }
                }
                free(v);
                free(d1);
            }
        }
}
