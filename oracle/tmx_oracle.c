/*
 * tmx_oracle.c -- CPU restatement of the reference T-mixer step (Tmixer.cpp).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA product is
 * checked against; nothing in the product links, loads or calls it.  It is
 * pinned bitwise against the reference itself (oracle/_ref, built by
 * oracle/build_ref.py) by tests/test_oracle_vs_ref.py.
 *
 * It restates, with runtime case parameters instead of compile-time #defines:
 *   GenerateInletVelocity          Tmixer.cpp:1426-1539
 *   initialization                 Tmixer.cpp:1544-1585
 *   equilibrium                    Tmixer.cpp:1589-1831
 *   initialize_distribution_function Tmixer.cpp:1835-2018
 *   boundary_conditions            Tmixer.cpp:2023-9033
 *   streaming                      Tmixer.cpp:9039-9347
 *   calculate_velocity_density     Tmixer.cpp:9352-9656
 *   collision                      Tmixer.cpp:9661-9860
 *   write_MixingQuality (numbers)  Tmixer.cpp:10161-10409
 *   write_Pressure_Power (numbers) Tmixer.cpp:9866-10027
 * with the same array semantics: two boxes (inlet "I" = box 0, mixing "M" =
 * box 1), each padded with ghost planes 0 and n+1 (allocated to n+2), z the
 * contiguous axis; four fields (flow f, species A g, B h, C p).
 *
 * Arithmetic follows the reference operation by operation (same grouping,
 * same true divisions, no fused multiply-add), so results are bit-identical.
 * Uninitialised "A*0" terms in the reference are taken as exact zeros.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int inx, iny, nz, mnx, mny, ia; /* ib = ia + mnx - 1 */
    double tau, taua, taub, taup;
    double rho0, rho_out, c0;
    double cin[3][2]; /* [species A,B,C][inlet 1,2]  (Tmixer.cpp:90-97) */
    double rateconst; /* Tmixer.cpp:99 */
    double umean;     /* mean of the inlet-1 duct profile, Tmixer.cpp:107 */
} orc_params;

typedef struct {
    orc_params P;
    int ib;
    int nx[2], ny[2], nz;
    size_t n[2];         /* padded node count per box */
    double *f[2][4][19]; /* post-stream / post-boundary populations */
    double *fn[2][4][19];/* post-collision populations */
    double *rho[2][4];   /* rho, grho, hrho, prho (mrho, ... in box 1) */
    double *u[2][3];
    double *uin1, *uin2; /* [(iny+3)][(nz+3)] */
    int steps;
} orc_t;

/* D3Q19 ordering, Tmixer.cpp:1368-1370 */
static const int EX[19] = {0, 1, 0, -1, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0};
static const int EY[19] = {0, 0, 1, 0, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1};
static const int EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};

static inline size_t IX(const orc_t *S, int b, int i, int j, int k)
{
    return ((size_t)i * (size_t)(S->ny[b] + 3) + (size_t)j) * (size_t)(S->nz + 3) + (size_t)k;
}
#define UIN(a, j, k) (a)[(size_t)(j) * (size_t)(S->nz + 3) + (size_t)(k)]

/* ------------------------------------------------------------------------ */
/* inlet profile: Tmixer.cpp:1426-1539                                       */
/* ------------------------------------------------------------------------ */
static void gen_inlet(orc_t *S)
{
    const int iny = S->P.iny, nz = S->P.nz;
    const double pi = 3.14159265358979323846;
    const double d = ((nz - 1.0) / 2.0);
    const double w = ((iny - 1.0) / 2.0);
    const double AR = (1.0 * w / d);
    const double twoARd = 2.0 * AR * d; /* (2.0*AR)*d */
    const double twod = 2.0 * d;
    const double ARAR = AR * AR;
    double *U1 = S->uin1, *U2 = S->uin2;
    for (int j = 0; j < iny; j++)
        for (int k = 0; k < nz; k++) {
            double nsum = 0;
            for (int n = 1; n <= 100; n++) {
                double msum = 0;
                for (int m = 1; m <= 100; m++) {
                    double N = (1.0 - cos(m * pi)) * (1.0 - cos(n * pi)) *
                               sin(((m * pi) / twoARd) * (j)) * sin(((n * pi) / twod) * (k));
                    double D = m * n * ((m * m) + (ARAR * n * n));
                    msum += (N / D);
                }
                nsum += msum;
            }
            UIN(U1, j + 1, k + 1) = nsum;
        }
    double sum = 0;
    for (int i = 1; i <= iny; i++)
        for (int j = 1; j <= nz; j++) sum += UIN(U1, i, j);
    double average = sum / ((iny) * (nz));
    for (int i = 1; i <= iny; i++)
        for (int j = 1; j <= nz; j++) UIN(U1, i, j) = UIN(U1, i, j) * (S->P.umean / average);
    for (int j = 0; j < iny; j++)
        for (int k = 0; k < nz; k++) {
            UIN(U1, j + 1, k) = UIN(U1, j + 1, k + 1);
            UIN(U2, j + 1, k + 2) = -UIN(U1, j + 1, k);
        }
    for (int i = 1; i <= iny; i++) {
        UIN(U1, i, 1) = 0;
        UIN(U2, i, nz) = 0;
    }
}

/* ------------------------------------------------------------------------ */
/* allocation and initialisation: Tmixer.cpp:711-1081, 1544-1585, 1835-2018 */
/* ------------------------------------------------------------------------ */
orc_t *orc_create(const orc_params *P)
{
    orc_t *S = (orc_t *)calloc(1, sizeof(orc_t));
    if (!S) return NULL;
    S->P = *P;
    S->ib = P->ia + P->mnx - 1;
    S->nx[0] = P->inx;
    S->ny[0] = P->iny;
    S->nx[1] = P->mnx;
    S->ny[1] = P->mny;
    S->nz = P->nz;
    for (int b = 0; b < 2; b++) {
        S->n[b] = (size_t)(S->nx[b] + 3) * (size_t)(S->ny[b] + 3) * (size_t)(S->nz + 3);
        for (int fl = 0; fl < 4; fl++) {
            for (int q = 0; q < 19; q++) {
                S->f[b][fl][q] = (double *)calloc(S->n[b], sizeof(double));
                S->fn[b][fl][q] = (double *)calloc(S->n[b], sizeof(double));
                if (!S->f[b][fl][q] || !S->fn[b][fl][q]) return NULL;
            }
            S->rho[b][fl] = (double *)calloc(S->n[b], sizeof(double));
            if (!S->rho[b][fl]) return NULL;
        }
        for (int a = 0; a < 3; a++) {
            S->u[b][a] = (double *)calloc(S->n[b], sizeof(double));
            if (!S->u[b][a]) return NULL;
        }
    }
    size_t nu = (size_t)(P->iny + 3) * (size_t)(P->nz + 3);
    S->uin1 = (double *)calloc(nu, sizeof(double));
    S->uin2 = (double *)calloc(nu, sizeof(double));
    if (!S->uin1 || !S->uin2) return NULL;
    return S;
}

void orc_destroy(orc_t *S)
{
    if (!S) return;
    for (int b = 0; b < 2; b++) {
        for (int fl = 0; fl < 4; fl++) {
            for (int q = 0; q < 19; q++) {
                free(S->f[b][fl][q]);
                free(S->fn[b][fl][q]);
            }
            free(S->rho[b][fl]);
        }
        for (int a = 0; a < 3; a++) free(S->u[b][a]);
    }
    free(S->uin1);
    free(S->uin2);
    free(S);
}

/* feq of one direction, Tmixer.cpp:1602-1830 (q=0: :1602; q=1..6 /18; q=7..18 /36) */
static inline double feq(double r, double ux, double uy, double uz, int q)
{
    double u2 = ux * ux + uy * uy + uz * uz;
    if (q == 0) return r * (1.0 - 3.0 * u2 / 2.0) / 3.0;
    double eu = ux * EX[q] + uy * EY[q] + uz * EZ[q];
    double poly = 1.0 + 3.0 * eu - 3.0 * u2 / 2.0 + 9.0 * eu * eu / 2.0;
    return (q <= 6) ? r * poly / 18.0 : r * poly / 36.0;
}

void orc_init(orc_t *S)
{
    gen_inlet(S);
    /* initialization(): every padded node */
    for (int b = 0; b < 2; b++)
        for (size_t x = 0; x < S->n[b]; x++) {
            S->rho[b][0][x] = S->P.rho0;
            S->rho[b][1][x] = S->P.c0;
            S->rho[b][2][x] = S->P.c0;
            S->rho[b][3][x] = S->P.c0;
            S->u[b][0][x] = 0;
            S->u[b][1][x] = 0;
            S->u[b][2][x] = 0;
        }
    /* equilibrium() then f = feq on padded nodes 0..n+1 */
    for (int b = 0; b < 2; b++)
        for (int i = 0; i <= S->nx[b] + 1; i++)
            for (int j = 0; j <= S->ny[b] + 1; j++)
                for (int k = 0; k <= S->nz + 1; k++) {
                    size_t x = IX(S, b, i, j, k);
                    for (int fl = 0; fl < 4; fl++)
                        for (int q = 0; q < 19; q++)
                            S->f[b][fl][q][x] =
                                feq(S->rho[b][fl][x], S->u[b][0][x], S->u[b][1][x], S->u[b][2][x], q);
                }
    S->steps = 0;
}

/* ------------------------------------------------------------------------ */
/* equilibrium + collision on padded nodes: Tmixer.cpp:1589-1831, 9661-9860  */
/* ------------------------------------------------------------------------ */
static void collide(orc_t *S)
{
    const double Ma = 1.0, Mb = 1.0, Mp = 2.0;
    const double w[19] = {1.0 / 3.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                          1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                          1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                          1.0 / 36.0};
    const double tf[4] = {S->P.tau, S->P.taua, S->P.taub, S->P.taup};
    for (int b = 0; b < 2; b++) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i <= S->nx[b] + 1; i++)
            for (int j = 0; j <= S->ny[b] + 1; j++)
                for (int k = 0; k <= S->nz + 1; k++) {
                    size_t x = IX(S, b, i, j, k);
                    double ux = S->u[b][0][x], uy = S->u[b][1][x], uz = S->u[b][2][x];
                    double Ca = S->rho[b][1][x] / Ma;
                    double Cb = S->rho[b][2][x] / Mb;
                    double rt = S->P.rateconst * Ca * Cb;
                    for (int fl = 0; fl < 4; fl++) {
                        double r = S->rho[b][fl][x];
                        double c1 = (1.0 - 1.0 / tf[fl]), c2 = (1.0 / tf[fl]);
                        for (int q = 0; q < 19; q++) {
                            double v = S->f[b][fl][q][x] * c1 + c2 * feq(r, ux, uy, uz, q);
                            if (fl == 1) v = v - w[q] * rt * Ma;
                            else if (fl == 2) v = v - w[q] * rt * Mb;
                            else if (fl == 3) v = v + w[q] * rt * Mp;
                            S->fn[b][fl][q][x] = v;
                        }
                    }
                }
    }
}

/* ------------------------------------------------------------------------ */
/* streaming, nodes 1..n of each box: Tmixer.cpp:9039-9347                   */
/* ------------------------------------------------------------------------ */
static void stream(orc_t *S)
{
    const int ia = S->P.ia, ib = S->ib, mny = S->P.mny;
    for (int b = 0; b < 2; b++) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 1; i <= S->nx[b]; i++)
            for (int j = 1; j <= S->ny[b]; j++)
                for (int k = 1; k <= S->nz; k++) {
                    size_t x = IX(S, b, i, j, k);
                    for (int fl = 0; fl < 4; fl++)
                        for (int q = 0; q < 19; q++) {
                            int si = i - EX[q], sj = j - EY[q], sk = k - EZ[q];
                            int sb = b;
                            /* inlet row 1 inside the opening pulls 2,7,8,15,18 from
                               mixing row mny (Tmixer.cpp:9077-9085) */
                            if (b == 0 && j == 1 && i >= ia && i <= ib && EY[q] == 1) {
                                sb = 1;
                                si = (i - ia + 1) - EX[q];
                                sj = mny;
                            }
                            /* mixing row mny pulls 4,9,10,16,17 from inlet row 1
                               (Tmixer.cpp:9230-9237) */
                            if (b == 1 && j == mny && EY[q] == -1) {
                                sb = 0;
                                si = (i + ia - 1) - EX[q];
                                sj = 1;
                            }
                            S->f[b][fl][q][x] = S->fn[sb][fl][q][IX(S, sb, si, sj, sk)];
                        }
                }
    }
}

/* ------------------------------------------------------------------------ */
/* moments: Tmixer.cpp:9352-9656                                             */
/* ------------------------------------------------------------------------ */
static void moments(orc_t *S)
{
    for (int b = 0; b < 2; b++)
        for (int fl = 0; fl < 4; fl++) memset(S->rho[b][fl], 0, S->n[b] * sizeof(double));
    for (int b = 0; b < 2; b++) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 1; i <= S->nx[b]; i++)
            for (int j = 1; j <= S->ny[b]; j++)
                for (int k = 1; k <= S->nz; k++) {
                    size_t x = IX(S, b, i, j, k);
                    for (int fl = 0; fl < 4; fl++) {
                        double s = S->f[b][fl][0][x];
                        for (int q = 1; q < 19; q++) s += S->f[b][fl][q][x];
                        S->rho[b][fl][x] = s;
                    }
                }
    }
    /* outlet row of the mixing box pinned to rho_out (Tmixer.cpp:9575-9582);
       the inlet ux forcing at :9565-9573 is overwritten below */
    for (int i = 1; i <= S->P.mnx; i++)
        for (int k = 1; k <= S->nz; k++) S->rho[1][0][IX(S, 1, i, 1, k)] = S->P.rho_out;
    for (int b = 0; b < 2; b++) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 1; i <= S->nx[b]; i++)
            for (int j = 1; j <= S->ny[b]; j++)
                for (int k = 1; k <= S->nz; k++) {
                    size_t x = IX(S, b, i, j, k);
                    double *const *f = S->f[b][0];
                    /* sums over index order 0..18; zero terms drop out exactly */
                    double sx = f[1][x] - f[3][x] + f[7][x] - f[8][x] - f[9][x] + f[10][x] +
                                f[11][x] - f[12][x] - f[13][x] + f[14][x];
                    double sy = f[2][x] - f[4][x] + f[7][x] + f[8][x] - f[9][x] - f[10][x] +
                                f[15][x] - f[16][x] - f[17][x] + f[18][x];
                    double sz = f[5][x] - f[6][x] + f[11][x] + f[12][x] - f[13][x] - f[14][x] +
                                f[15][x] + f[16][x] - f[17][x] - f[18][x];
                    double r = S->rho[b][0][x];
                    S->u[b][0][x] = sx / r;
                    S->u[b][1][x] = sy / r;
                    S->u[b][2][x] = sz / r;
                }
    }
}

/* ------------------------------------------------------------------------ */
/* boundary conditions: Tmixer.cpp:2023-9033                                 */
/* ------------------------------------------------------------------------ */
/* Every case below works on one node of one field at a time: the node's 19
 * post-stream populations are loaded into v[], the closure runs, v[] is
 * stored back.  Fields never read each other inside a closure, so running the
 * four fields of a node together matches the reference's field-by-field loops.
 * Density arrays ("R") are the reference's rho/grho/hrho/prho: at this point
 * they hold the previous step's moments, overwritten in place by the cases
 * that write them, exactly as in the reference. */
typedef struct {
    orc_t *S;
    int b, fl;
    size_t x;
    double v[19];
} nd_t;

static inline void ld(nd_t *N, orc_t *S, int b, int fl, int i, int j, int k)
{
    N->S = S;
    N->b = b;
    N->fl = fl;
    N->x = IX(S, b, i, j, k);
    for (int q = 0; q < 19; q++) N->v[q] = S->f[b][fl][q][N->x];
}
static inline void st(nd_t *N)
{
    for (int q = 0; q < 19; q++) N->S->f[N->b][N->fl][q][N->x] = N->v[q];
}
/* own post-collision population ("undo streaming") */
static inline double FN(const nd_t *N, int q) { return N->S->fn[N->b][N->fl][q][N->x]; }
/* density array of the node's field at another node of the same box */
static inline double *RP(const nd_t *N, int i, int j, int k)
{
    return &N->S->rho[N->b][N->fl][IX(N->S, N->b, i, j, k)];
}
static inline double *RSELF(const nd_t *N) { return &N->S->rho[N->b][N->fl][N->x]; }
/* rho = f0 + f1 + ... + f18 in index order */
static inline double s19(const double *v)
{
    double s = v[0];
    for (int q = 1; q < 19; q++) s += v[q];
    return s;
}
/* the same sum without directions a and c */
static inline double sx2(const double *v, int a, int c)
{
    double s = 0;
    int first = 1;
    for (int q = 0; q < 19; q++) {
        if (q == a || q == c) continue;
        if (first) {
            s = v[q];
            first = 0;
        } else
            s += v[q];
    }
    return s;
}
/* species zero-gradient copy of all 19 populations from another node */
static inline void copy19(nd_t *N, int b, int i, int j, int k)
{
    size_t y = IX(N->S, b, i, j, k);
    for (int q = 0; q < 19; q++) N->v[q] = N->S->f[b][N->fl][q][y];
}

#define V N->v

/* --- inlet-box edges along x with an undo-averaged buried pair ----------- */
/* Case 2 (Tmixer.cpp:2030-2186) and Case 3 (:2187-2342): y=1, z=nz */
static void cl_edge_y1_ztop(nd_t *N)
{
    V[2] = V[4];
    V[6] = V[5];
    V[7] = V[9];
    V[8] = V[10];
    V[13] = V[11];
    V[14] = V[12];
    V[18] = V[16];
    V[15] = (1.0 / 2.0) * (FN(N, 15) + FN(N, 17));
    V[17] = V[15];
    *RSELF(N) = s19(V);
    double A = (1.0 / 4.0) * (V[1] - V[3]);
    V[7] = V[9] - A;
    V[8] = V[10] + A;
    V[13] = V[11] + A;
    V[14] = V[12] - A;
}
/* Case 20 (:4238-4385): y=iny, z=nz */
static void cl_edge_ytop_ztop(nd_t *N)
{
    V[4] = V[2];
    V[6] = V[5];
    V[9] = V[7];
    V[10] = V[8];
    V[13] = V[11];
    V[14] = V[12];
    V[17] = V[15];
    V[16] = (1.0 / 2.0) * (FN(N, 16) + FN(N, 18));
    V[18] = V[16];
    *RSELF(N) = s19(V);
    double A = (1.0 / 4.0) * (V[1] - V[3]);
    V[9] = V[7] + A;
    V[10] = V[8] - A;
    V[13] = V[11] + A;
    V[14] = V[12] - A;
}
/* Case 21 (:4386-4533): y=iny, z=1 */
static void cl_edge_ytop_z1(nd_t *N)
{
    V[4] = V[2];
    V[5] = V[6];
    V[9] = V[7];
    V[10] = V[8];
    V[11] = V[13];
    V[12] = V[14];
    V[16] = V[18];
    V[15] = (1.0 / 2.0) * (FN(N, 15) + FN(N, 17));
    V[17] = V[15];
    *RSELF(N) = s19(V);
    double A = (1.0 / 4.0) * (V[1] - V[3]);
    V[9] = V[7] + A;
    V[10] = V[8] - A;
    V[11] = V[13] - A;
    V[12] = V[14] + A;
}
/* Case 28 (:5282-5425) and Case 29 (:5426-5571): y=1, z=1 */
static void cl_edge_y1_z1(nd_t *N)
{
    V[2] = V[4];
    V[5] = V[6];
    V[7] = V[9];
    V[8] = V[10];
    V[11] = V[13];
    V[12] = V[14];
    V[15] = V[17];
    V[16] = (1.0 / 2.0) * (FN(N, 16) + FN(N, 18));
    V[18] = V[16];
    *RSELF(N) = s19(V);
    double A = (1.0 / 4.0) * (V[1] - V[3]);
    V[7] = V[9] - A;
    V[8] = V[10] + A;
    V[11] = V[13] - A;
    V[12] = V[14] + A;
}

/* --- inlet-box edges closed from a neighbour's density ------------------- */
/* Case 4 (:2343-2476): x=1, z=nz; density from (1, j, nz-1).  For field C the
   reference assigns g13 instead of p13 (:2474), so p13 keeps its undo-streamed
   value. */
static void cl_edge_x1_ztop(nd_t *N, int j)
{
    const int nz = N->S->nz;
    double B = 1.0 / 4.0 * (V[2] - V[4]);
    V[1] = V[3];
    V[6] = V[5];
    V[7] = V[9] - B;
    V[10] = V[8] + B;
    V[14] = V[12];
    V[17] = V[15] + B;
    V[18] = V[16] - B;
    V[11] = FN(N, 11);
    V[13] = FN(N, 13);
    V[11] = (1.0 / 2.0) * (*RP(N, 1, j, nz - 1) - sx2(V, 11, 13));
    if (N->fl != 3) V[13] = V[11];
}
/* Case 6 (:2477-2605): x=inx, z=nz; density from (inx, j, nz-1) */
static void cl_edge_xtop_ztop(nd_t *N, int j)
{
    const int nz = N->S->nz, inx = N->S->P.inx;
    double B = (1.0 / 4.0) * (V[2] - V[4]);
    V[3] = V[1];
    V[6] = V[5];
    V[9] = V[7] + B;
    V[8] = V[10] - B;
    V[13] = V[11];
    V[17] = V[15] + B;
    V[18] = V[16] - B;
    V[12] = (1.0 / 2.0) * (*RP(N, inx, j, nz - 1) - sx2(V, 12, 14));
    V[14] = V[12];
}
/* Case 22 (:4534-4656): x=1, z=1; density from (1, j, 2) */
static void cl_edge_x1_z1(nd_t *N, int j)
{
    double B = 1.0 / 4.0 * (V[2] - V[4]);
    V[1] = V[3];
    V[5] = V[6];
    V[7] = V[9] - B;
    V[10] = V[8] + B;
    V[11] = V[13];
    V[15] = V[17] - B;
    V[16] = V[18] + B;
    V[12] = (1.0 / 2.0) * (*RP(N, 1, j, 2) - sx2(V, 12, 14));
    V[14] = V[12];
}
/* Case 23 (:4657-4779): x=inx, z=1; density from (inx, j, 2) */
static void cl_edge_xtop_z1(nd_t *N, int j)
{
    const int inx = N->S->P.inx;
    double B = 1.0 / 4.0 * (V[2] - V[4]);
    V[3] = V[1];
    V[5] = V[6];
    V[8] = V[10] - B;
    V[9] = V[7] + B;
    V[12] = V[14];
    V[15] = V[17] - B;
    V[16] = V[18] + B;
    V[11] = (1.0 / 2.0) * (*RP(N, inx, j, 2) - sx2(V, 11, 13));
    V[13] = V[11];
}
/* Case 24 (:4780-4909): x=1, y=1; density from (1, 2, k) */
static void cl_edge_x1_y1(nd_t *N, int k)
{
    double C = 1.0 / 4.0 * (V[5] - V[6]);
    V[1] = V[3];
    V[2] = V[4];
    V[7] = V[9];
    V[11] = V[13] - C;
    V[14] = V[12] + C;
    V[15] = V[17] - C;
    V[18] = V[16] + C;
    V[8] = (1.0 / 2.0) * (*RP(N, 1, 2, k) - sx2(V, 8, 10));
    V[10] = V[8];
}
/* Case 25 (:4910-5032): x=1, y=iny; density from (1, iny-1, k) */
static void cl_edge_x1_ytop(nd_t *N, int k)
{
    const int iny = N->S->P.iny;
    double C = 1.0 / 4.0 * (V[5] - V[6]);
    V[1] = V[3];
    V[4] = V[2];
    V[10] = V[8];
    V[11] = V[13] - C;
    V[14] = V[12] + C;
    V[16] = V[18] - C;
    V[17] = V[15] + C;
    V[7] = (1.0 / 2.0) * (*RP(N, 1, iny - 1, k) - sx2(V, 7, 9));
    V[9] = V[7];
}
/* Case 26 (:5033-5159): x=inx, y=1; density from (inx, 2, k) */
static void cl_edge_xtop_y1(nd_t *N, int k)
{
    const int inx = N->S->P.inx;
    double C = 1.0 / 4.0 * (V[5] - V[6]);
    V[3] = V[1];
    V[2] = V[4];
    V[8] = V[10];
    V[12] = V[14] - C;
    V[13] = V[11] + C;
    V[15] = V[17] - C;
    V[18] = V[16] + C;
    V[7] = (1.0 / 2.0) * (*RP(N, inx, 2, k) - sx2(V, 7, 9));
    V[9] = V[7];
}
/* Case 27 (:5160-5281): x=inx, y=iny; density from (inx, iny-1, k) */
static void cl_edge_xtop_ytop(nd_t *N, int k)
{
    const int inx = N->S->P.inx, iny = N->S->P.iny;
    double C = 1.0 / 4.0 * (V[5] - V[6]);
    V[3] = V[1];
    V[4] = V[2];
    V[9] = V[7];
    V[12] = V[14] - C;
    V[13] = V[11] + C;
    V[16] = V[18] - C;
    V[17] = V[15] + C;
    V[8] = (1.0 / 2.0) * (*RP(N, inx, iny - 1, k) - sx2(V, 8, 10));
    V[10] = V[8];
}

/* --- velocity inlets (Zou-He type) and species Dirichlet inlets --------- */
/* Inlet1 flow (:2606-2626) */
static void cl_inlet1_flow(nd_t *N, double U)
{
    double r = (1.0 / (1.0 - U)) * ((V[0] + V[2] + V[4] + V[5] + V[6] + V[15] + V[16] + V[17] + V[18]) +
                                    2.0 * (V[3] + V[8] + V[9] + V[12] + V[13]));
    *RSELF(N) = r;
    double A = (-r * U) / 6.0;
    double B = (1.0 / 2.0) * (V[2] - V[4] + V[15] - V[16] - V[17] + V[18]);
    double C = (1.0 / 2.0) * (V[5] - V[6] + V[15] + V[16] - V[17] - V[18]);
    V[1] = V[3] + (r * U) / 3.0;
    V[7] = V[9] - (A + B);
    V[10] = V[8] - (A - B);
    V[11] = V[13] - (A + C);
    V[14] = V[12] - (A - C);
}
/* Inlet1 species (:2627-2666): anti-bounce-back to the inlet concentration */
static void cl_inlet1_species(nd_t *N, double c)
{
    V[1] = -V[3] + (2.0 / 18.0) * c;
    V[7] = -V[9] + (2.0 / 36.0) * c;
    V[10] = -V[8] + (2.0 / 36.0) * c;
    V[11] = -V[13] + (2.0 / 36.0) * c;
    V[14] = -V[12] + (2.0 / 36.0) * c;
}
/* Inlet2 flow (:2668-2690) */
static void cl_inlet2_flow(nd_t *N, double U)
{
    double r = (1.0 / (1.0 + (U))) * ((V[0] + V[2] + V[4] + V[5] + V[6] + V[15] + V[16] + V[17] + V[18]) +
                                      2.0 * (V[1] + V[7] + V[10] + V[11] + V[14]));
    *RSELF(N) = r;
    double A = (-r * (U)) / 6.0;
    double B = (1.0 / 2.0) * (V[2] - V[4] + V[15] - V[16] - V[17] + V[18]);
    double C = (1.0 / 2.0) * (V[5] - V[6] + V[15] + V[16] - V[17] - V[18]);
    V[3] = V[1] - (r * (U)) / 3.0;
    V[9] = V[7] + (A + B);
    V[8] = V[10] + (A - B);
    V[13] = V[11] + (A + C);
    V[12] = V[14] + (A - C);
}
/* Inlet2 species (:2691-2730) */
static void cl_inlet2_species(nd_t *N, double c)
{
    V[3] = -V[1] + (2.0 / 18.0) * c;
    V[9] = -V[7] + (2.0 / 36.0) * c;
    V[8] = -V[10] + (2.0 / 36.0) * c;
    V[13] = -V[11] + (2.0 / 36.0) * c;
    V[12] = -V[14] + (2.0 / 36.0) * c;
}

/* --- no-slip faces (flow) --------------------------------------------- */
/* Case 10 (:2731-2764): inlet box y=iny */
static void cl_face_ytop(nd_t *N)
{
    double C = (1.0 / 2.0) * (V[5] - V[6] + V[11] + V[12] - V[13] - V[14]);
    V[4] = V[2];
    V[16] = V[18] - C;
    V[17] = V[15] + C;
    V[9] = V[7];
    V[10] = V[8];
    *RSELF(N) = s19(V);
    double A = (1.0 / 2.0) * (V[1] - V[3] + V[11] - V[12] - V[13] + V[14]);
    V[9] = V[7] + A;
    V[10] = V[8] - A;
}
/* Case 11 (:2874-2906) and Case 12 (:3016-3049): inlet box y=1 walls */
static void cl_face_y1(nd_t *N)
{
    double C = (1.0 / 2.0) * (V[5] - V[6] + V[11] + V[12] - V[13] - V[14]);
    V[2] = V[4];
    V[15] = V[17] - C;
    V[18] = V[16] + C;
    V[7] = V[9];
    V[8] = V[10];
    *RSELF(N) = s19(V);
    double A = (1.0 / 2.0) * (V[1] - V[3] + V[11] - V[12] - V[13] + V[14]);
    V[7] = V[9] - A;
    V[8] = V[10] + A;
}
/* Case 13 (:3162-3190): outlet, pressure rho_out; writes no density */
static void cl_outlet(nd_t *N, double rout)
{
    double uy = 1.0 - (1.0 / rout) * ((V[0] + V[1] + V[3] + V[5] + V[6] + V[11] + V[12] + V[13] + V[14]) +
                                      2.0 * (V[4] + V[9] + V[10] + V[16] + V[17]));
    double A = (rout * uy) / 6.0;
    double B = (1.0 / 2.0) * ((V[3] + V[12] + V[13]) - (V[1] + V[11] + V[14]));
    double C = (1.0 / 2.0) * ((V[6] + V[13] + V[14]) - (V[5] + V[11] + V[12]));
    V[2] = V[4] + (rout * uy) / 3.0;
    V[7] = V[9] + (A + B);
    V[8] = V[10] + (A - B);
    V[15] = V[17] + (A + C);
    V[18] = V[16] + (A - C);
}
/* Case 14 (:3275-3310): mixing box x=1 */
static void cl_face_mx1(nd_t *N)
{
    double C = (1.0 / 2.0) * ((V[6] + V[17] + V[18]) - (V[5] + V[15] + V[16]));
    V[1] = V[3];
    V[11] = V[13] + (C);
    V[14] = V[12] - (C);
    V[7] = V[9];
    V[10] = V[8];
    *RSELF(N) = s19(V);
    double A = (1.0 / 2.0) * ((V[2] + V[15] + V[18]) - (V[4] + V[16] + V[17]));
    V[7] = V[9] - A;
    V[10] = V[8] + A;
}
/* Case 15 (:3405-3439): mixing box x=mnx */
static void cl_face_mxtop(nd_t *N)
{
    double C = (1.0 / 2.0) * ((V[6] + V[17] + V[18]) - (V[5] + V[15] + V[16]));
    V[3] = V[1];
    V[13] = V[11] - (C);
    V[12] = V[14] + (C);
    V[9] = V[7];
    V[8] = V[10];
    *RSELF(N) = s19(V);
    double A = (1.0 / 2.0) * ((V[2] + V[15] + V[18]) - (V[4] + V[16] + V[17]));
    V[9] = V[7] + A;
    V[8] = V[10] - A;
}
/* Case 16 (:3540-3569) and Case 17 (:3666-3721): z=nz faces */
static void cl_face_ztop(nd_t *N)
{
    double B = (1.0 / 2.0) * (V[2] - V[4] + V[7] + V[8] - V[9] - V[10]);
    V[6] = V[5];
    V[17] = V[15] + B;
    V[18] = V[16] - B;
    V[13] = V[11];
    V[14] = V[12];
    *RSELF(N) = s19(V);
    double A = (1.0 / 2.0) * (V[1] - V[3] + V[7] - V[8] - V[9] + V[10]);
    V[13] = V[11] + A;
    V[14] = V[12] - A;
}
/* Case 18 (:3888-3919) and Case 19 (:4010-4065): z=1 faces */
static void cl_face_z1(nd_t *N)
{
    double B = (1.0 / 2.0) * (V[2] - V[4] + V[7] + V[8] - V[9] - V[10]);
    V[5] = V[6];
    V[15] = V[17] - B;
    V[16] = V[18] + B;
    V[11] = V[13];
    V[12] = V[14];
    *RSELF(N) = s19(V);
    double A = (1.0 / 2.0) * (V[1] - V[3] + V[7] - V[8] - V[9] + V[10]);
    V[11] = V[13] - A;
    V[12] = V[14] + A;
}

/* --- corners (:5572-7785) ------------------------------------------------ */
/* A corner bounces back six populations, sets two buried pairs to the average
 * of their own post-collision values, and (except at the junction corners)
 * closes a third pair from a density.  bb[6][2] = {to, from}; avg[3][2] pairs
 * (the first entry receives 0.5*(fn_a + fn_b), the second copies it); cpair =
 * {to, copy} of the density-closed pair or {-1,-1}; R = the density used. */
typedef struct {
    int bb[6][2];
    int navg;
    int avg[3][2];
    int cpair[2];
} corner_t;

static void cl_corner(nd_t *N, const corner_t *c, double R)
{
    for (int t = 0; t < 6; t++) V[c->bb[t][0]] = V[c->bb[t][1]];
    double fa[3];
    for (int t = 0; t < c->navg; t++) fa[t] = (1.0 / 2.0) * (FN(N, c->avg[t][0]) + FN(N, c->avg[t][1]));
    for (int t = 0; t < c->navg; t++) {
        V[c->avg[t][0]] = fa[t];
        V[c->avg[t][1]] = fa[t];
    }
    if (c->cpair[0] >= 0) {
        V[c->cpair[0]] = (1.0 / 2.0) * (R - sx2(V, c->cpair[0], c->cpair[1]));
        V[c->cpair[1]] = V[c->cpair[0]];
    }
}

/* Corner 1 G' (1,iny,nz) :5580 ... Corner 16 D (ia,1,1) :7661 */
static const corner_t CORNER[16] = {
    /* 1 G' */ {{{1, 3}, {4, 2}, {6, 5}, {10, 8}, {14, 12}, {17, 15}}, 2, {{9, 7}, {11, 13}}, {16, 18}},
    /* 2 F' */ {{{3, 1}, {4, 2}, {6, 5}, {17, 15}, {13, 11}, {9, 7}}, 2, {{10, 8}, {12, 14}}, {16, 18}},
    /* 3 H' */ {{{1, 3}, {2, 4}, {6, 5}, {7, 9}, {18, 16}, {14, 12}}, 2, {{10, 8}, {11, 13}}, {15, 17}},
    /* 4 E' */ {{{3, 1}, {2, 4}, {6, 5}, {8, 10}, {13, 11}, {18, 16}}, 2, {{9, 7}, {12, 14}}, {15, 17}},
    /* 5 G  */ {{{1, 3}, {4, 2}, {5, 6}, {16, 18}, {11, 13}, {10, 8}}, 2, {{9, 7}, {14, 12}}, {15, 17}},
    /* 6 F  */ {{{3, 1}, {4, 2}, {5, 6}, {9, 7}, {12, 14}, {16, 18}}, 2, {{10, 8}, {11, 13}}, {15, 17}},
    /* 7 H  */ {{{1, 3}, {2, 4}, {5, 6}, {7, 9}, {11, 13}, {15, 17}}, 2, {{10, 8}, {12, 14}}, {16, 18}},
    /* 8 E  */ {{{3, 1}, {2, 4}, {5, 6}, {8, 10}, {12, 14}, {15, 17}}, 2, {{9, 7}, {11, 13}}, {16, 18}},
    /* 9 A  */ {{{1, 3}, {2, 4}, {5, 6}, {7, 9}, {11, 13}, {15, 17}}, 2, {{10, 8}, {12, 14}}, {16, 18}},
    /*10 B  */ {{{3, 1}, {2, 4}, {5, 6}, {8, 10}, {12, 14}, {15, 17}}, 2, {{9, 7}, {11, 13}}, {16, 18}},
    /*11 A' */ {{{1, 3}, {2, 4}, {6, 5}, {7, 9}, {18, 16}, {14, 12}}, 2, {{10, 8}, {11, 13}}, {15, 17}},
    /*12 B' */ {{{3, 1}, {2, 4}, {6, 5}, {8, 10}, {13, 11}, {18, 16}}, 2, {{9, 7}, {12, 14}}, {15, 17}},
    /*13 D' */ {{{6, 5}, {7, 9}, {13, 11}, {14, 12}, {17, 15}, {18, 16}}, 3, {{1, 3}, {4, 2}, {8, 10}}, {-1, -1}},
    /*14 C' */ {{{6, 5}, {8, 10}, {13, 11}, {14, 12}, {17, 15}, {18, 16}}, 3, {{9, 7}, {4, 2}, {1, 3}}, {-1, -1}},
    /*15 C  */ {{{5, 6}, {8, 10}, {11, 13}, {12, 14}, {15, 17}, {16, 18}}, 3, {{1, 3}, {4, 2}, {9, 7}}, {-1, -1}},
    /*16 D  */ {{{5, 6}, {7, 9}, {11, 13}, {12, 14}, {15, 17}, {16, 18}}, 3, {{1, 3}, {4, 2}, {8, 10}}, {-1, -1}},
};

/* --- mixing-box edges (:7786-8550) ------------------------------------- */
/* Edge AB (:7788-7868): y=1, z=1; pair 16/18 from rho_out (flow) or the
   species density at (i, 2, 1) */
static void cl_medge_y1_z1(nd_t *N, double R)
{
    double A = (1.0 / 4.0) * (V[1] - V[3]);
    V[2] = V[4];
    V[5] = V[6];
    V[7] = V[9] - A;
    V[8] = V[10] + A;
    V[11] = V[13] - A;
    V[12] = V[14] + A;
    V[15] = V[17];
    V[18] = (1.0 / 2.0) * (R - sx2(V, 16, 18));
    V[16] = V[18];
}
/* Edge A'B' (:7870-7950): y=1, z=nz; pair 15/17 */
static void cl_medge_y1_ztop(nd_t *N, double R)
{
    double A = (1.0 / 4.0) * (V[1] - V[3]);
    V[2] = V[4];
    V[6] = V[5];
    V[7] = V[9] - A;
    V[8] = V[10] + A;
    V[13] = V[11] + A;
    V[14] = V[12] - A;
    V[18] = V[16];
    V[15] = (1.0 / 2.0) * (R - sx2(V, 15, 17));
    V[17] = V[15];
}
/* Edge AA' (:7951-8043): x=1, y=1; pair 8/10 */
static void cl_medge_x1_y1(nd_t *N, double R)
{
    double C = (1.0 / 4.0) * (V[5] - V[6]);
    V[1] = V[3];
    V[2] = V[4];
    V[7] = V[9];
    V[11] = V[13] - C;
    V[14] = V[12] + C;
    V[15] = V[17] - C;
    V[18] = V[16] + C;
    V[8] = (1.0 / 2.0) * (R - sx2(V, 8, 10));
    V[10] = V[8];
}
/* Edge BB' (:8044-8136): x=mnx, y=1; pair 7/9 */
static void cl_medge_xtop_y1(nd_t *N, double R)
{
    double C = (1.0 / 4.0) * (V[5] - V[6]);
    V[3] = V[1];
    V[2] = V[4];
    V[8] = V[10];
    V[12] = V[14] - C;
    V[13] = V[11] + C;
    V[15] = V[17] - C;
    V[18] = V[16] + C;
    V[7] = (1.0 / 2.0) * (R - sx2(V, 7, 9));
    V[9] = V[7];
}
/* Edge AD (:8137-8244): x=1, z=1; buried 12/14 averaged */
static void cl_medge_x1_z1(nd_t *N)
{
    double B = (1.0 / 4.0) * (V[2] - V[4]);
    V[1] = V[3];
    V[5] = V[6];
    V[7] = V[9] - B;
    V[10] = V[8] + B;
    V[11] = V[13];
    V[15] = V[17] - B;
    V[16] = V[18] + B;
    V[14] = (1.0 / 2.0) * (FN(N, 12) + FN(N, 14));
    V[12] = V[14];
}
/* Edge A'D' (:8245-8344): x=1, z=nz; buried 11/13 averaged */
static void cl_medge_x1_ztop(nd_t *N)
{
    double B = (1.0 / 4.0) * (V[2] - V[4]);
    V[1] = V[3];
    V[6] = V[5];
    V[7] = V[9] - B;
    V[10] = V[8] + B;
    V[14] = V[12];
    V[17] = V[15] + B;
    V[18] = V[16] - B;
    V[13] = (1.0 / 2.0) * (FN(N, 11) + FN(N, 13));
    V[11] = V[13];
}
/* Edge BC (:8345-8445): x=mnx, z=1; buried 11/13 averaged */
static void cl_medge_xtop_z1(nd_t *N)
{
    double B = (1.0 / 4.0) * (V[2] - V[4]);
    V[3] = V[1];
    V[5] = V[6];
    V[8] = V[10] - B;
    V[9] = V[7] + B;
    V[12] = V[14];
    V[15] = V[17] - B;
    V[16] = V[18] + B;
    V[13] = (1.0 / 2.0) * (FN(N, 11) + FN(N, 13));
    V[11] = V[13];
}
/* Edge B'C' (:8446-8550): x=mnx, z=nz; buried 12/14 averaged */
static void cl_medge_xtop_ztop(nd_t *N)
{
    double B = (1.0 / 4.0) * (V[2] - V[4]);
    V[3] = V[1];
    V[6] = V[5];
    V[9] = V[7] + B;
    V[8] = V[10] - B;
    V[13] = V[11];
    V[17] = V[15] + B;
    V[18] = V[16] - B;
    V[14] = (1.0 / 2.0) * (FN(N, 12) + FN(N, 14));
    V[12] = V[14];
}

/* --- junction edges DD' (:8551-8792) and CC' (:8793-9033) ---------------- */
/* every population but the rest one and the closed pair is restored to its
   own post-collision value and averaged with its opposite; the closed pair
   comes from the density at (x, 2, k) */
static void cl_junction_edge(nd_t *N, int x, int k, int closed, int closed_copy)
{
    static const int pairs_dd[8][2] = {{3, 1}, {4, 2}, {6, 5}, {10, 8}, {13, 11}, {14, 12}, {17, 15}, {18, 16}};
    static const int pairs_cc[8][2] = {{3, 1}, {4, 2}, {6, 5}, {9, 7}, {13, 11}, {14, 12}, {17, 15}, {18, 16}};
    const int(*pairs)[2] = (closed == 7) ? pairs_dd : pairs_cc;
    for (int t = 0; t < 8; t++) {
        double a = (1.0 / 2.0) * (FN(N, pairs[t][0]) + FN(N, pairs[t][1]));
        V[pairs[t][0]] = a;
        V[pairs[t][1]] = a;
    }
    V[closed] = (1.0 / 2.0) * (*RP(N, x, 2, k) - sx2(V, closed, closed_copy));
    V[closed_copy] = V[closed];
}

#undef V

/* run a closure over a node set for all four fields */
#define FOR_FIELDS(b, i, j, k, STMT)                                                                \
    for (int fl = 0; fl < 4; fl++) {                                                                \
        nd_t N_;                                                                                    \
        nd_t *N = &N_;                                                                              \
        ld(N, S, b, fl, i, j, k);                                                                   \
        STMT;                                                                                       \
        st(N);                                                                                      \
    }

static void boundary(orc_t *S)
{
    const int inx = S->P.inx, iny = S->P.iny, nz = S->P.nz, mnx = S->P.mnx, mny = S->P.mny;
    const int ia = S->P.ia, ib = S->ib;
    const double rout = S->P.rho_out;
    int i, j, k;

    /* Case 2, Case 3 */
    for (i = 2; i <= ia - 1; i++) FOR_FIELDS(0, i, 1, nz, cl_edge_y1_ztop(N));
    for (i = ib + 1; i <= inx - 1; i++) FOR_FIELDS(0, i, 1, nz, cl_edge_y1_ztop(N));
    /* Case 4, Case 6 */
    for (j = 2; j <= iny - 1; j++) FOR_FIELDS(0, 1, j, nz, cl_edge_x1_ztop(N, j));
    for (j = 2; j <= iny - 1; j++) FOR_FIELDS(0, inx, j, nz, cl_edge_xtop_ztop(N, j));
    /* Inlet1, Inlet2 */
    for (j = 2; j <= iny - 1; j++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(0, 1, j, k,
                       if (fl == 0) cl_inlet1_flow(N, UIN(S->uin1, j, k));
                       else cl_inlet1_species(N, S->P.cin[fl - 1][0]));
    for (j = 2; j <= iny - 1; j++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(0, inx, j, k,
                       if (fl == 0) cl_inlet2_flow(N, UIN(S->uin2, j, k));
                       else cl_inlet2_species(N, S->P.cin[fl - 1][1]));
    /* Case 10: y=iny */
    for (i = 2; i <= inx - 1; i++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(0, i, iny, k, if (fl == 0) cl_face_ytop(N); else copy19(N, 0, i, iny - 1, k));
    /* Case 11, Case 12: y=1 walls */
    for (i = 2; i <= ia - 1; i++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(0, i, 1, k, if (fl == 0) cl_face_y1(N); else copy19(N, 0, i, 2, k));
    for (i = ib + 1; i <= inx - 1; i++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(0, i, 1, k, if (fl == 0) cl_face_y1(N); else copy19(N, 0, i, 2, k));
    /* Case 13: outlet */
    for (i = 2; i <= mnx - 1; i++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(1, i, 1, k, if (fl == 0) cl_outlet(N, rout); else copy19(N, 1, i, 2, k));
    /* Case 14, Case 15 */
    for (j = 2; j <= mny; j++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(1, 1, j, k, if (fl == 0) cl_face_mx1(N); else copy19(N, 1, 2, j, k));
    for (j = 2; j <= mny; j++)
        for (k = 2; k <= nz - 1; k++)
            FOR_FIELDS(1, mnx, j, k, if (fl == 0) cl_face_mxtop(N); else copy19(N, 1, mnx - 1, j, k));
    /* Case 16: inlet box z=nz */
    for (i = 2; i <= inx - 1; i++)
        for (j = 2; j <= iny - 1; j++)
            FOR_FIELDS(0, i, j, nz, if (fl == 0) cl_face_ztop(N); else copy19(N, 0, i, j, nz - 1));
    /* Case 17: mixing box z=nz, rows 2..mny+1; row mny+1 also closes the
       inlet opening node (i+ia-1, 1, nz) */
    for (i = 2; i <= mnx - 1; i++)
        for (j = 2; j <= mny + 1; j++) {
            FOR_FIELDS(1, i, j, nz, if (fl == 0) cl_face_ztop(N); else copy19(N, 1, i, j, nz - 1));
            if (j == mny + 1)
                FOR_FIELDS(0, i + ia - 1, 1, nz,
                           if (fl == 0) cl_face_ztop(N); else copy19(N, 0, i + ia - 1, 1, nz - 1));
        }
    /* Case 18: inlet box z=1 */
    for (i = 2; i <= inx - 1; i++)
        for (j = 2; j <= iny - 1; j++)
            FOR_FIELDS(0, i, j, 1, if (fl == 0) cl_face_z1(N); else copy19(N, 0, i, j, 2));
    /* Case 19: mixing box z=1 (+ inlet opening node at z=1) */
    for (i = 2; i <= mnx - 1; i++)
        for (j = 2; j <= mny + 1; j++) {
            FOR_FIELDS(1, i, j, 1, if (fl == 0) cl_face_z1(N); else copy19(N, 1, i, j, 2));
            if (j == mny + 1)
                FOR_FIELDS(0, i + ia - 1, 1, 1, if (fl == 0) cl_face_z1(N); else copy19(N, 0, i + ia - 1, 1, 2));
        }
    /* Cases 20..29 */
    for (i = 2; i <= inx - 1; i++) FOR_FIELDS(0, i, iny, nz, cl_edge_ytop_ztop(N));
    for (i = 2; i <= inx - 1; i++) FOR_FIELDS(0, i, iny, 1, cl_edge_ytop_z1(N));
    for (j = 2; j <= iny - 1; j++) FOR_FIELDS(0, 1, j, 1, cl_edge_x1_z1(N, j));
    for (j = 2; j <= iny - 1; j++) FOR_FIELDS(0, inx, j, 1, cl_edge_xtop_z1(N, j));
    for (k = 2; k <= nz - 1; k++) FOR_FIELDS(0, 1, 1, k, cl_edge_x1_y1(N, k));
    for (k = 2; k <= nz - 1; k++) FOR_FIELDS(0, 1, iny, k, cl_edge_x1_ytop(N, k));
    for (k = 2; k <= nz - 1; k++) FOR_FIELDS(0, inx, 1, k, cl_edge_xtop_y1(N, k));
    for (k = 2; k <= nz - 1; k++) FOR_FIELDS(0, inx, iny, k, cl_edge_xtop_ytop(N, k));
    for (i = 2; i <= ia - 1; i++) FOR_FIELDS(0, i, 1, 1, cl_edge_y1_z1(N));
    for (i = ib + 1; i <= inx - 1; i++) FOR_FIELDS(0, i, 1, 1, cl_edge_y1_z1(N));

    /* corners 1..8: inlet box; density from the adjacent x-y edge node */
    {
        const int cx[8] = {1, inx, 1, inx, 1, inx, 1, inx};
        const int cy[8] = {iny, iny, 1, 1, iny, iny, 1, 1};
        const int cz[8] = {nz, nz, nz, nz, 1, 1, 1, 1};
        for (int c = 0; c < 8; c++) {
            int rz = (cz[c] == nz) ? nz - 1 : 2;
            FOR_FIELDS(0, cx[c], cy[c], cz[c], cl_corner(N, &CORNER[c], *RP(N, cx[c], cy[c], rz)));
        }
    }
    /* corners 9..12: outlet corners; flow closes from rho_out, the species
       from their density one row below the outlet (ghost row 0) */
    {
        const int cx[4] = {1, mnx, 1, mnx};
        const int cz[4] = {1, 1, nz, nz};
        for (int c = 0; c < 4; c++)
            FOR_FIELDS(1, cx[c], 1, cz[c],
                       cl_corner(N, &CORNER[8 + c], (fl == 0) ? rout : *RP(N, cx[c], 0, cz[c])));
    }
    /* corners 13..16: junction corners, no density closure */
    {
        const int cx[4] = {ia, ib, ib, ia};
        const int cz[4] = {nz, nz, 1, 1};
        for (int c = 0; c < 4; c++) FOR_FIELDS(0, cx[c], 1, cz[c], cl_corner(N, &CORNER[12 + c], 0.0));
    }
    /* mixing-box edges */
    for (i = 2; i <= mnx - 1; i++)
        FOR_FIELDS(1, i, 1, 1, cl_medge_y1_z1(N, (fl == 0) ? rout : *RP(N, i, 2, 1)));
    for (i = 2; i <= mnx - 1; i++)
        FOR_FIELDS(1, i, 1, nz, cl_medge_y1_ztop(N, (fl == 0) ? rout : *RP(N, i, 2, nz)));
    for (k = 2; k <= nz - 1; k++)
        FOR_FIELDS(1, 1, 1, k, cl_medge_x1_y1(N, (fl == 0) ? rout : *RP(N, 1, 2, k)));
    for (k = 2; k <= nz - 1; k++)
        FOR_FIELDS(1, mnx, 1, k, cl_medge_xtop_y1(N, (fl == 0) ? rout : *RP(N, mnx, 2, k)));
    for (j = 2; j <= mny; j++) FOR_FIELDS(1, 1, j, 1, cl_medge_x1_z1(N));
    for (j = 2; j <= mny; j++) FOR_FIELDS(1, 1, j, nz, cl_medge_x1_ztop(N));
    for (j = 2; j <= mny; j++) FOR_FIELDS(1, mnx, j, 1, cl_medge_xtop_z1(N));
    for (j = 2; j <= mny; j++) FOR_FIELDS(1, mnx, j, nz, cl_medge_xtop_ztop(N));
    /* junction edges DD' (x=ia) and CC' (x=ib) */
    for (k = 2; k <= nz - 1; k++) FOR_FIELDS(0, ia, 1, k, cl_junction_edge(N, ia, k, 7, 9));
    for (k = 2; k <= nz - 1; k++) FOR_FIELDS(0, ib, 1, k, cl_junction_edge(N, ib, k, 8, 10));
}

/* ------------------------------------------------------------------------ */
/* public entry points                                                       */
/* ------------------------------------------------------------------------ */
void orc_step(orc_t *S, int nsteps)
{
    for (int s = 0; s < nsteps; s++) {
        collide(S);
        stream(S);
        boundary(S);
        moments(S);
        S->steps++;
    }
}

/* field: 0 rho, 1 ux, 2 uy, 3 uz, 4 cA, 5 cB, 6 cC; nodes 1..n, k fastest */
void orc_fields(const orc_t *S, int box, int field, double *out)
{
    size_t o = 0;
    const double *a = (field == 0) ? S->rho[box][0] : (field <= 3) ? S->u[box][field - 1] : S->rho[box][field - 3];
    for (int i = 1; i <= S->nx[box]; i++)
        for (int j = 1; j <= S->ny[box]; j++)
            for (int k = 1; k <= S->nz; k++) out[o++] = a[IX(S, box, i, j, k)];
}

/* post-step population q of field fl, nodes 1..n */
void orc_pops(const orc_t *S, int box, int fl, int q, double *out)
{
    size_t o = 0;
    for (int i = 1; i <= S->nx[box]; i++)
        for (int j = 1; j <= S->ny[box]; j++)
            for (int k = 1; k <= S->nz; k++) out[o++] = S->f[box][fl][q][IX(S, box, i, j, k)];
}

void orc_inlet_profile(const orc_t *S, double *u1, double *u2)
{
    size_t n = (size_t)(S->P.iny + 3) * (size_t)(S->P.nz + 3);
    memcpy(u1, S->uin1, n * sizeof(double));
    memcpy(u2, S->uin2, n * sizeof(double));
}

/* Mixing quality, Tmixer.cpp:10161-10409 (the numbers it prints): one row per
 * mixing row j=1..mny then per inlet row j=1..iny over x=ia..ib; each row is
 * {j, cA mean, cB mean, cC mean, IA, IB, IC}.  The running maxima start at 0. */
void orc_mixing(const orc_t *S, double *rows)
{
    const int nz = S->nz, mnx = S->P.mnx, mny = S->P.mny, iny = S->P.iny;
    double mx[3] = {0, 0, 0};
    for (int part = 0; part < 2; part++) {
        int b = part == 0 ? 1 : 0;
        int nrow = part == 0 ? mny : iny;
        int i0 = part == 0 ? 1 : S->P.ia, i1 = part == 0 ? mnx : S->ib;
        for (int j = 1; j <= nrow; j++) {
            double avg[3], var[3];
            for (int s = 0; s < 3; s++) {
                const double *c = S->rho[b][s + 1];
                double sumx = 0;
                for (int i = i0; i <= i1; i++) {
                    double sumz = 0;
                    for (int k = 1; k <= nz; k++) {
                        double v = c[IX(S, b, i, j, k)];
                        sumz += v;
                        if (mx[s] < v) mx[s] = v;
                    }
                    sumx += sumz;
                }
                avg[s] = (sumx / (1.0 * nz * mnx));
            }
            for (int s = 0; s < 3; s++) {
                const double *c = S->rho[b][s + 1];
                double sumx = 0;
                for (int i = i0; i <= i1; i++) {
                    double sumz = 0;
                    for (int k = 1; k <= nz; k++) {
                        double dlt = c[IX(S, b, i, j, k)] - avg[s];
                        sumz += pow(dlt, 2.0);
                    }
                    sumx += sumz;
                }
                var[s] = (1.0 / (1.0 * nz * mnx)) * sumx;
            }
            double *r = rows + 7 * (size_t)(part == 0 ? (j - 1) : (mny + j - 1));
            r[0] = part == 0 ? j : j + mny;
            r[1] = avg[0];
            r[2] = avg[1];
            r[3] = avg[2];
            int ok = part == 0 ? (avg[0] > 0 && avg[1] > 0 && avg[2] > 0) : (avg[0] > 0);
            for (int s = 0; s < 3; s++) {
                if (ok) {
                    double Is = var[s] / (avg[s] * (mx[s] - avg[s]));
                    r[4 + s] = (part == 0 ? 1 : 1.0) - sqrt(Is);
                } else
                    r[4 + s] = 0.0;
            }
        }
    }
}

/* Pressure and specific power, Tmixer.cpp:9866-10027 (the numbers it prints),
 * in lattice units, with the reference's unit factors:
 *   prow[(mny+iny)*3]  {row, p, p - p_top}: p = mean density / 3 over mixing
 *                      row j=1..mny (x=1..mnx), then inlet row j=1..iny
 *                      (x=ia..ib, divided by nz*mnx as the reference does);
 *                      p_top = the same over inlet row iny (:9895-9905)
 *   px[inx*2]          {i, p}: mean density / 3 over the inlet cross-section x=i
 *   pw[(mny-2)*5]      {j, cross-section rate, total rate, the same two summed
 *                      over every column}: for j=2..mny-1 the reference's loop
 *                      (:9985-10024) assigns the per-column rates inside the
 *                      x loop, so only column mnx-1 reaches the k sums; the
 *                      last two entries add every column instead
 *   units[2]           P0 and Pw0 (Tmixer.cpp:189-196), the factors the
 *                      reference multiplies the printed values by */
void orc_pressure_power(const orc_t *S, double *prow, double *px, double *pw, double *units)
{
    const int nz = S->nz, mnx = S->P.mnx, mny = S->P.mny, iny = S->P.iny, inx = S->P.inx, ia = S->P.ia;
    const double *ri = S->rho[0][0], *rm = S->rho[1][0];
    const double *ux = S->u[1][0], *uy = S->u[1][1], *uz = S->u[1][2];
    const double tau = S->P.tau, rho0 = S->P.rho0;
    /* unit factors as the reference's macros expand (length = inx) */
    const double L0 = (0.0008 / (inx - 1));
    const double T0 = ((((2.0 * tau - 1.0) / 6.0) / 0.000001004) * (L0 * L0));
    const double M0 = ((101325.0 / (rho0 / 3.0)) * (L0 * T0 * T0));
    units[0] = ((M0) / (L0 * T0 * T0));
    units[1] = ((L0 * L0) / (T0 * T0 * T0));
    const double vis = ((2.0 * tau - 1.0) / 6.0) * (1.0 * 1.0 * 1.0);

    double sumx = 0;
    for (int i = 1; i <= mnx; i++) {
        double sumz = 0;
        for (int k = 1; k <= nz; k++) sumz += ri[IX(S, 0, i + ia - 1, iny, k)];
        sumx += sumz;
    }
    const double ptop = (sumx / (1.0 * nz * mnx)) / 3.0;
    for (int j = 1; j <= mny; j++) {
        sumx = 0;
        for (int i = 1; i <= mnx; i++) {
            double sumz = 0;
            for (int k = 1; k <= nz; k++) sumz += rm[IX(S, 1, i, j, k)];
            sumx += sumz;
        }
        const double t = (sumx / (1.0 * nz * mnx)) / 3.0;
        double *r = prow + 3 * (size_t)(j - 1);
        r[0] = j;
        r[1] = t;
        r[2] = t - ptop;
    }
    for (int j = 1; j <= iny; j++) {
        sumx = 0;
        for (int i = ia; i <= S->ib; i++) {
            double sumz = 0;
            for (int k = 1; k <= nz; k++) sumz += ri[IX(S, 0, i, j, k)];
            sumx += sumz;
        }
        const double t = (sumx / (1.0 * nz * mnx)) / 3.0;
        double *r = prow + 3 * (size_t)(mny + j - 1);
        r[0] = j + mny;
        r[1] = t;
        r[2] = t - ptop;
    }
    for (int i = 1; i <= inx; i++) {
        double sumy = 0;
        for (int j = 1; j <= iny; j++) {
            double sumz = 0;
            for (int k = 1; k <= nz; k++) sumz += ri[IX(S, 0, i, j, k)];
            sumy += sumz;
        }
        px[2 * (size_t)(i - 1)] = i;
        px[2 * (size_t)(i - 1) + 1] = (sumy / (1.0 * nz * iny)) / 3.0;
    }
    for (int j = 2; j < mny; j++) {
        double sumz = 0, sumtotalz = 0, allz = 0, alltotalz = 0;
        for (int k = 2; k < nz; k++) {
            double sx = 0, stx = 0, allx = 0, alltx = 0;
            for (int i = 2; i < mnx; i++) {
#define M_(a, ii, jj, kk) a[IX(S, 1, ii, jj, kk)]
                const double delux = (M_(ux, i + 1, j, k) - M_(ux, i - 1, j, k)) / 2.0;
                const double delvy = (M_(uy, i, j + 1, k) - M_(uy, i, j - 1, k)) / 2.0;
                const double delwz = (M_(uz, i, j, k + 1) - M_(uz, i, j, k - 1)) / 2.0;
                const double deluy = (M_(ux, i, j + 1, k) - M_(ux, i, j - 1, k)) / 2.0;
                const double delvx = (M_(uy, i + 1, j, k) - M_(uy, i - 1, j, k)) / 2.0;
                const double deluz = (M_(ux, i, j, k + 1) - M_(ux, i, j, k - 1)) / 2.0;
                const double delwx = (M_(uz, i + 1, j, k) - M_(uz, i - 1, j, k)) / 2.0;
                const double delvz = (M_(uy, i, j, k + 1) - M_(uy, i, j, k - 1)) / 2.0;
                const double delwy = (M_(uz, i, j + 1, k) - M_(uz, i, j - 1, k)) / 2.0;
#undef M_
                sx = pow(delux, 2.0) + pow(delwz, 2.0) + 0.5 * pow((deluz + delwx), 2.0);
                stx = pow(delux, 2.0) + pow(delvy, 2.0) + pow(delwz, 2.0) + 0.5 * pow((delvx + deluy), 2.0) +
                      0.5 * pow((deluz + delwx), 2.0) + 0.5 * pow((delvz + delwy), 2.0);
                allx += sx;
                alltx += stx;
            }
            sumz += sx;
            sumtotalz += stx;
            allz += allx;
            alltotalz += alltx;
        }
        double *r = pw + 5 * (size_t)(j - 2);
        r[0] = j;
        r[1] = 2.0 * vis * (sumz / (1.0 * (nz - 2) * (mnx - 2)));
        r[2] = 2.0 * vis * (sumtotalz / (1.0 * (nz - 2) * (mnx - 2)));
        r[3] = 2.0 * vis * (allz / (1.0 * (nz - 2) * (mnx - 2)));
        r[4] = 2.0 * vis * (alltotalz / (1.0 * (nz - 2) * (mnx - 2)));
    }
}

int orc_steps_done(const orc_t *S) { return S->steps; }

/* The post-collision populations the next step would stream (the next
 * step's equilibrium + collision, Tmixer.cpp:1589-1831 and :9661-9860),
 * left in the fn arrays; the next orc_step recomputes them identically. */
void orc_collide_preview(orc_t *S) { collide(S); }

/* post-collision population q of field fl after orc_collide_preview */
void orc_fn(const orc_t *S, int box, int fl, int q, double *out)
{
    size_t o = 0;
    for (int i = 1; i <= S->nx[box]; i++)
        for (int j = 1; j <= S->ny[box]; j++)
            for (int k = 1; k <= S->nz; k++) out[o++] = S->fn[box][fl][q][IX(S, box, i, j, k)];
}
