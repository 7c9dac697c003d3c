/*
 * liberi_oracle.c -- CPU restatement of libERI's RHF Fock build.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * engine in gms_liberi_b200/.  Only the tests, the smoke check and the CPU
 * baseline leg of bench.py load it; the product never links or calls it.
 *
 * What is restated (line-faithful to the reference's behaviour):
 *   - shell classification into ascending per-L shell lists
 *       (src/liberi_shell_pair.F90:137-346, final sort :301-344)
 *   - the six pair classes ss,sp,pp,sd,pd,dd: pair order, packed Schwarz lookup,
 *     primitive-pair data and the mu*R^2 > cux=50 "ismlp" flag
 *       (src/liberi_shell_pair.F90:348-1283, e.g. compute_ss_pairs :348-474)
 *   - the 21 s/p/d kernels in the driver's fixed order
 *       (src/liberi_driver.F90:69-102), then the 34 f kernels of the ENABLE_F
 *       block in its order (src/liberi_driver.F90:103-160): four f pair
 *       classes sf, pf, df, ff (src/liberi_shell_pair.F90:1285-1682; lower-L
 *       shell outer, f inner, ff triangular), GAMESS f order xxx, yyy, zzz,
 *       xxy, xxz, xyy, yyz, xzz, yzz, xyz with sqrt5 on the six mixed and
 *       sqrt15 on xyz (int3011_rysgen.F90 ijx/ijy/ijz, d03bra)
 *     with each kernel's own pre-screen (cross-class or own-class maxima),
 *     product test operator (>=, > or none), bra-range / flat-index rank split
 *     with its tile size, and digestion cut
 *       (src/rhf/rot_axis/int0000.F90:58-107, int0001.F90:67-121,
 *        int2211_rysgen.F90:295-356, int2222_rysgen.F90:393-431, ...)
 *   - DIRFCK digestion with the GAMESS unique-component loops (iandj, kandl,
 *     same), index sorting, 0.5 factors and the six packed updates
 *       (src/rhf/rot_axis/int0000.F90:241-311, int1111.F90:1894-2020,
 *        int2222_rysgen.F90:11176-11338)
 *
 * Integral values.  The reference evaluates (ab|cd) with rotated-axis Boys-table
 * kernels (s/p/d up to L=5) and generated Rys kernels (L>=5 with a d-d pair).
 * Both are exact methods up to ~1e-14; this oracle evaluates every class by Rys
 * quadrature.  Rys classes take the reference's own root algorithm: the
 * discretised Stieltjes procedure (RYSDS) on Gauss-Legendre nodes u=t^2 --
 * 30 points for up to 4 roots (int2111_rysgen.F90:473-533), 35 for 5
 * (int2222_rysgen.F90:661-697), 40 for 6 and 7 (int3333_rysgen.F90:1229-1309)
 * -- followed by the Golub-Welsch step (the reference's RYSGW, below),
 * int2222_rysgen.F90:636-877.  The ERIC kernels of the f block (int0030,
 * int0031, int0032, int1030: src/rhf/eric/) work from tabulated Boys
 * functions like the rotated-axis ones (int0030_ericgen.F90:261-300) and are
 * restated the same way, without their primitive skip.  Rotated-axis classes work, like the reference's,
 * from tabulated Boys functions (liberi_boys.F90): the Rys rule is formed from
 * the Boys moments F_0..F_{2n-1} in long double.
 * The asymptotic branch follows the reference per class: rotated-axis classes
 * switch to the large-T form for T > t_max = 25 (src/liberi_boys.F90:22,
 * int0000.F90:220-234), Rys classes for xx >= 43 / 49 / 55 / 60 / 65 (3 / 4 /
 * 5 / 6 / 7 roots, int2111_rysgen.F90:458, int2211_rysgen.F90:540,
 * int2222_rysgen.F90:642, int3322_rysgen.F90, int3333_rysgen.F90:1206).
 * The large-T Boys form sqrt(pi/4t)*(2m-1)!!/(2t)^m is exactly the Gauss-
 * Hermite limit of the Rys roots, so both branches are reproduced.
 *
 * Deliberate deviations (both far below the 1e-10 parity bar):
 *   - d_coeff_alt / sq for primitive pairs with mu*R^2 > 50 are left
 *     uninitialised by the reference (liberi_shell_pair.F90:438-441); here the
 *     Rys and ERIC classes use the formula value, the rotated-axis classes skip
 *     the pair as the reference does (int0000.F90:208-210).
 *   - the reference decodes triangular pair indices in single precision for
 *     most kernels (int0001.F90:124); here the decode is exact integer math,
 *     which agrees for every pair count below ~2M.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Scalar types of the quartet arithmetic (roots, recurrences, assembly,
 * digestion): double and long double in this build.  The op-counting build
 * (oracle/opcount.cpp) compiles this file as C++ with a counting type in
 * their place, to measure the floating-point operations per primitive and
 * per shell quartet of this restatement of the reference algorithm. */
#ifndef ORACLE_REAL
#define ORACLE_REAL double
#define ORACLE_REALL long double
#define ORACLE_OPS() 0
#define ORACLE_MARK()
#define ORACLE_MARKED() 0
#endif
typedef ORACLE_REAL real_t;
typedef ORACLE_REALL reall_t;

#define PI_D 3.14159265358979323846
#define MAXGRID 40
#define MAXROOT 7
#define MAXCART 10
#define MAXL 3
#define NK 55  /* 21 s/p/d kernels, then the 34 of the f block */

/* ---- reference parameters (src/liberi_parameters.F90) -------------------- */
static const double CUX = 50.0;                   /* :44 */

/* ---- Cartesian component tables: p = x,y,z ; d = xx,yy,zz,xy,xz,yz ;
 * f = xxx,yyy,zzz,xxy,xxz,xyy,yyz,xzz,yzz,xyz ----------------------------- */
static const int NCART[4] = {1, 3, 6, 10};
static const int CX[4][10] = {{0}, {1, 0, 0}, {2, 0, 0, 1, 1, 0}, {3, 0, 0, 2, 2, 1, 0, 1, 0, 1}};
static const int CY[4][10] = {{0}, {0, 1, 0}, {0, 2, 0, 1, 0, 1}, {0, 3, 0, 1, 0, 2, 2, 0, 1, 1}};
static const int CZ[4][10] = {{0}, {0, 0, 1}, {0, 0, 2, 0, 1, 1}, {0, 0, 3, 0, 1, 0, 1, 2, 2, 1}};
/* off-diagonal d components carry sqrt(3) (int2222_rysgen.F90:599-634), the
 * six mixed f components sqrt(5) and xyz sqrt(15) (int3011_rysgen.F90 d03bra) */
static double CNORM[4][10];

/* ---- input basis (mirror of basis_t, src/liberi_types.f90:26-67) --------- */
typedef struct {
    int32_t nsh, natoms, num_bas, mxgtot;
    const int32_t *ang_mom;   /* 1=s 2=p 3=d 4=f */
    const int32_t *contr_num;
    const int32_t *sh_loc;    /* 1-based primitive offset */
    const int32_t *atom_num;  /* 1-based */
    const int32_t *atom_loc;  /* 1-based first basis function */
    const double *exponents;
    const double *coef_s, *coef_p, *coef_d, *coef_f;
    const double *coords;     /* 3*natoms */
    const double *schwrz;     /* nsh(nsh+1)/2 packed */
} oracle_basis;

typedef struct {
    double schwarz_cut;  /* reference cutoff_schwarz (5e-11 literal) */
    double eri_cut;      /* reference literal 5.0d-11 in most digestions */
    int32_t my_rank, num_procs;
    int32_t sample_mod;  /* >1: evaluate only the quartets of a hashed 1/sample_mod of bra pairs */
    int32_t sample_seed;
    int32_t nthreads;
    int32_t only_kernel; /* -1: all, else kernel index 0..NK-1 */
} oracle_opts;

/* per kernel: [0] screened shell quartets, [1] primitive quartets evaluated,
 * [2] integrals digested (|v| >= cut), [3] evaluated shell quartets (sample);
 * t_wall[k]: wall seconds of the kernel, t_eval[k]: seconds spent evaluating
 * and digesting quartets summed over threads; fp[k]: fingerprint of the
 * screened-quartet set owned by this rank, {sum, xor} over its quartets of
 * quartet_fp() (order independent, so any evaluation order gives the same
 * pair of words; the engine computes the same function over its task lists) */
typedef struct {
    int64_t c[NK][4];
    double t_wall[NK];
    double t_eval[NK];
    int32_t nthreads;
    uint64_t fp[NK][2];
    uint64_t ops[NK][2];  /* op-counting build only: ops in primitive-quartet work, in shell-quartet work */
} oracle_counts;

/* ---- pair classes: the six s/p/d ones, then sf, pf, df, ff ----------------- */
enum { SS = 0, SP, PP, SD, PD, DD, SF, PF, DF, FF, NPC };
static const int PC_L1[NPC] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
static const int PC_L2[NPC] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};

typedef struct {
    int64_t n;          /* shell pairs */
    int32_t *ish, *jsh; /* 0-based shells (first, second) */
    double *xint;
    int64_t *loc;       /* n+1 primitive-pair offsets */
    double *ea, *eb, *cc;  /* exponents, c_a*c_b */
    int32_t *ismlp;
} pairs_t;

typedef struct {
    const oracle_basis *b;
    double (*csh)[3];     /* shell coordinates */
    int32_t *lst[MAXL + 1];  /* ascending shell lists per L */
    int64_t nl[MAXL + 1];
    pairs_t pc[NPC];
    const double *coef[MAXL + 1];
} ctx_t;

/* ---- kernel descriptors (src/liberi_driver.F90:69-160) ------------------- */
enum { OP_GE = 0, OP_GT = 1, OP_NONE = 2 };
enum { TILE_SQRT = 0, TILE_E9 = 1, TILE_E8 = 2, TILE_NONE = 3 };
/* rys: Rys root algorithm (discretised Stieltjes on ngrid points), else the
 * Boys-function rule (rotated-axis and ERIC kernels); skip: primitive pairs
 * with mu R^2 > 50 skipped (rotated-axis kernels only) */
typedef struct {
    const char *name;
    int bra, ket, tri, rys, cross, op, tile, ketmajor, digest_schwarz;
    double asym;  /* rot: T > 25 ; rys: xx >= asym */
    int ngrid, skip;
} kdesc_t;

static const kdesc_t KD[NK] = {
    /* name      bra ket tri rys cross op      tile       kmaj dsch asym grid skip */
    {"int0000", SS, SS, 1, 0, 0, OP_GE, TILE_SQRT, 0, 1, 25.0, 0, 1},
    {"int0001", SS, SP, 0, 0, 1, OP_GT, TILE_E9, 0, 1, 25.0, 0, 1},
    {"int0011", SS, PP, 0, 0, 1, OP_GT, TILE_E9, 0, 1, 25.0, 0, 1},
    {"int0111", SP, PP, 0, 0, 1, OP_GT, TILE_E9, 0, 0, 25.0, 0, 1},
    {"int0101", SP, SP, 1, 0, 0, OP_GE, TILE_NONE, 0, 0, 25.0, 0, 1},
    {"int1111", PP, PP, 1, 0, 0, OP_GE, TILE_NONE, 0, 1, 25.0, 0, 1},
    {"int0002", SS, SD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int0012", SS, PD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int0102", SP, SD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int0112", SP, PD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int0022", SS, DD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int0122", SP, DD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int1102", PP, SD, 0, 0, 1, OP_GT, TILE_E8, 0, 0, 25.0, 0, 1},
    {"int0202", SD, SD, 1, 0, 0, OP_GT, TILE_NONE, 0, 0, 25.0, 0, 1},
    {"int2211", DD, PP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int2121", PD, PD, 1, 1, 0, OP_GT, TILE_NONE, 0, 0, 49.0, 30, 0},
    {"int2120", PD, SD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 43.0, 30, 0},
    {"int2111", PD, PP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 43.0, 30, 0},
    {"int2220", DD, SD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int2221", DD, PD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int2222", DD, DD, 1, 1, 0, OP_NONE, TILE_NONE, 0, 0, 55.0, 35, 0},
    /* f block: own-class pre-screens, ">" product test except int3333 (none),
     * 3.75e8 tiles for product kernels, bra-fastest flat order in the Rys
     * product kernels and bra-major in the ERIC ones (int0030_ericgen.F90:
     * 66-124, int3011_rysgen.F90:213-274, int3333_rysgen.F90:829-867);
     * digestion at the literal 5e-11 throughout */
    {"int3333", FF, FF, 1, 1, 0, OP_NONE, TILE_NONE, 0, 0, 65.0, 40, 0},
    {"int0030", SS, SF, 0, 0, 0, OP_GT, TILE_E8, 0, 0, 25.0, 0, 0},
    {"int0031", SS, PF, 0, 0, 0, OP_GT, TILE_E8, 0, 0, 25.0, 0, 0},
    {"int0032", SS, DF, 0, 0, 0, OP_GT, TILE_E8, 0, 0, 25.0, 0, 0},
    {"int1030", SP, SF, 0, 0, 0, OP_GT, TILE_E8, 0, 0, 25.0, 0, 0},
    {"int3330", FF, SF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3011", SF, PP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 43.0, 30, 0},
    {"int3020", SF, SD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 43.0, 30, 0},
    {"int2130", PD, SF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int2230", DD, SF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3030", SF, SF, 1, 1, 0, OP_GT, TILE_NONE, 0, 0, 49.0, 30, 0},
    {"int3110", PF, SP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 43.0, 30, 0},
    {"int3111", PF, PP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3120", PF, SD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3121", PF, PD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int2231", DD, PF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3130", PF, SF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3131", PF, PF, 1, 1, 0, OP_GT, TILE_NONE, 0, 0, 55.0, 35, 0},
    {"int3210", DF, SP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3331", FF, PF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 60.0, 40, 0},
    {"int3211", DF, PP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3220", DF, SD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3221", DF, PD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3222", DF, DD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3230", DF, SF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3231", DF, PF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3232", DF, DF, 1, 1, 0, OP_GT, TILE_NONE, 0, 0, 60.0, 40, 0},
    {"int3300", FF, SS, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3310", FF, SP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 49.0, 30, 0},
    {"int3311", FF, PP, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3320", FF, SD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3321", FF, PD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 55.0, 35, 0},
    {"int3322", FF, DD, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 60.0, 40, 0},
    {"int3332", FF, DF, 0, 1, 0, OP_GT, TILE_E8, 1, 0, 60.0, 40, 0},
};

/* ======================= Rys roots and weights ============================= */
/* Gauss-Legendre grids of the RYSDS procedure: 30, 35 and 40 points */
static double GRID_U[3][MAXGRID], GRID_W[3][MAXGRID];
static int grid_slot(int ngrid) { return ngrid <= 30 ? 0 : (ngrid <= 35 ? 1 : 2); }
/* asymptotic: u_i = HR[n][i]/T, w_i = HW[n][i]/sqrt(T) (Gauss-Hermite, 2n pts) */
static double HR[MAXROOT + 1][MAXROOT], HW[MAXROOT + 1][MAXROOT];
static int g_init = 0;

/* Gauss-Legendre nodes on [-1,1] by Newton on P_n */
static void gauss_legendre(int n, double *x, double *w) {
    for (int i = 0; i < n; i++) {
        double z = cos(PI_D * (i + 0.75) / (n + 0.5)), pp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

/* eigenvalues of a symmetric tridiagonal (diag a[0..n-1], offdiag^2 b[1..n-1])
 * by Sturm-count bisection, ascending; eigen-weights via Christoffel numbers. */
static int sturm_count(int n, const double *a, const double *b2, double x) {
    int cnt = 0;
    double q = a[0] - x;
    if (q < 0) cnt++;
    for (int i = 1; i < n; i++) {
        if (q == 0.0) q = 1e-300;
        q = a[i] - x - b2[i] / q;
        if (q < 0) cnt++;
    }
    return cnt;
}

static void jacobi_gauss(int n, const double *a, const double *b2, double beta0,
                         double lo, double hi, double *x, double *w) {
    for (int k = 0; k < n; k++) {
        double l = lo, h = hi;
        for (int it = 0; it < 200; it++) {
            double m = 0.5 * (l + h);
            if (m == l || m == h) break;
            if (sturm_count(n, a, b2, m) > k) h = m; else l = m;
        }
        double xr = 0.5 * (l + h);
        /* Christoffel: w = beta0 / sum_k p_k(x)^2 / (b2_1...b2_k) with
         * normalised recurrence */
        double p0 = 1.0, p1 = 0.0, s = 1.0, nrm = 1.0;
        for (int j = 0; j < n - 1; j++) {
            double pn = (xr - a[j]) * p0 - (j > 0 ? b2[j] * p1 : 0.0);
            p1 = p0;
            p0 = pn;
            nrm *= b2[j + 1];
            s += p0 * p0 / nrm;
        }
        x[k] = xr;
        w[k] = beta0 / s;
    }
}

/* ---- rotated-axis classes: Boys functions and the Rys rule from them ------
 * The reference's rotated-axis kernels work from tabulated Boys functions
 * F_m(T) for T <= t_max = 25 (src/liberi_boys.F90:22-32) and the large-T form
 * beyond.  Here F_m is tabulated as a Taylor table (step 0.05, nine terms,
 * long double) and the Gauss rule of the Rys weight, whose moments are
 * exactly F_0..F_{2n-1}, is formed from those moments by the Chebyshev
 * algorithm in long double (n <= 3 for these classes). */
#define BOYS_STEP 0.05L
#define BOYS_NPT 503
#define BOYS_MMAX 14
#define BOYS_TERMS 9
static long double BOYS[BOYS_NPT][BOYS_MMAX + 1];
static double BOYS_D[BOYS_NPT][BOYS_MMAX + 1];

static void boys_table_init(void) {
    for (int k = 0; k < BOYS_NPT; k++) {
        long double T = k * BOYS_STEP, e = expl(-T);
        /* series for the highest order, downward recursion for the rest */
        long double term = 1.0L / (2 * BOYS_MMAX + 1), s = term;
        for (int j = 1; j < 400; j++) {
            term *= 2.0L * T / (2 * BOYS_MMAX + 2 * j + 1);
            s += term;
            if (term < 1e-30L * s) break;
        }
        BOYS[k][BOYS_MMAX] = e * s;
        for (int m = BOYS_MMAX; m > 0; m--) BOYS[k][m - 1] = (2.0L * T * BOYS[k][m] + e) / (2 * m - 1);
        for (int m = 0; m <= BOYS_MMAX; m++) BOYS_D[k][m] = (double)BOYS[k][m];
    }
}

/* double-precision Rys rule for 1 and 2 roots (well conditioned) */
static void rys_small_d(int n, real_t T, real_t *u, real_t *w) {
    const int mmax = 2 * n - 1;
    const int k = (int)((double)T / (double)BOYS_STEP + 0.5);
    const real_t d = T - k * (double)BOYS_STEP;
    real_t F[4], sm = 0.0, f = 1.0;
    for (int j = 0; j < BOYS_TERMS; j++) {
        sm += BOYS_D[k][mmax + j] * f;
        f *= -d / (double)(j + 1);
    }
    F[mmax] = sm;
    const real_t e = exp(-T);
    for (int m = mmax; m > 0; m--) F[m - 1] = (2.0 * T * F[m] + e) / (double)(2 * m - 1);
    if (n == 1) {
        u[0] = F[1] / F[0];
        w[0] = F[0];
        return;
    }
    /* monic recurrence from the moments, then the 2x2 Jacobi matrix */
    const real_t a0 = F[1] / F[0];
    const real_t s1 = F[2] - a0 * F[1], s2 = F[3] - a0 * F[2];  /* sigma_{1,1}, sigma_{1,2} */
    const real_t b1 = s1 / F[0];
    const real_t a1 = s2 / s1 - a0;
    const real_t m = 0.5 * (a0 + a1), h = 0.5 * (a1 - a0), r = sqrt(h * h + b1);
    const real_t x0 = m - r, x1 = m + r;
    u[0] = x0;
    u[1] = x1;
    w[0] = F[0] / (1.0 + (x0 - a0) * (x0 - a0) / b1);
    w[1] = F[0] / (1.0 + (x1 - a0) * (x1 - a0) / b1);
}

/* F_0..F_mmax(T), T <= 25 */
static void boys_eval(int mmax, real_t T, reall_t *F) {
    int k = (int)((long double)(double)T / BOYS_STEP + 0.5L);
    reall_t d = (reall_t)T - k * BOYS_STEP;
    reall_t sm = 0.0L, f = 1.0L;
    for (int j = 0; j < BOYS_TERMS; j++) {
        sm += BOYS[k][mmax + j] * f;
        f *= -d / (long double)(j + 1);
    }
    F[mmax] = sm;
    reall_t e = expl(-(reall_t)T);
    for (int m = mmax; m > 0; m--) F[m - 1] = (2.0L * (reall_t)T * F[m] + e) / (long double)(2 * m - 1);
}

/* Gauss rule (n <= 3) of the Rys weight from its moments F_0..F_{2n-1} */
static void rys_from_moments(int n, real_t T, real_t *u, real_t *w) {
    reall_t F[2 * MAXROOT + 1];
    boys_eval(2 * n - 1, T, F);
    reall_t a[MAXROOT], b[MAXROOT];
    reall_t sp[2 * MAXROOT], sc[2 * MAXROOT], sn[2 * MAXROOT];
    for (int l = 0; l < MAXROOT; l++) { a[l] = 0.0L; b[l] = 0.0L; }
    for (int l = 0; l < 2 * MAXROOT; l++) { sp[l] = 0.0L; sn[l] = 0.0L; }
    for (int l = 0; l < 2 * n; l++) sc[l] = F[l];
    a[0] = F[1] / F[0];
    b[0] = F[0];
    for (int k = 1; k < n; k++) {
        for (int l = k; l < 2 * n - k; l++) sn[l] = sc[l + 1] - a[k - 1] * sc[l] - b[k - 1] * sp[l];
        a[k] = sn[k + 1] / sn[k] - sc[k] / sc[k - 1];
        b[k] = sn[k] / sc[k - 1];
        for (int l = 0; l < 2 * n; l++) { sp[l] = sc[l]; sc[l] = sn[l]; }
    }
    reall_t x[MAXROOT];
    if (n == 1) {
        x[0] = a[0];
    } else if (n == 2) {
        reall_t m = 0.5L * (a[0] + a[1]), h = 0.5L * (a[1] - a[0]);
        reall_t r = sqrtl(h * h + b[1]);
        x[0] = m - r;
        x[1] = m + r;
    } else {
        /* characteristic polynomial of the 3x3 Jacobi matrix, trigonometric
         * roots, two Newton polishing steps each */
        reall_t c2 = -(a[0] + a[1] + a[2]);
        reall_t c1 = a[0] * a[1] + a[0] * a[2] + a[1] * a[2] - b[1] - b[2];
        reall_t c0 = -(a[0] * a[1] * a[2]) + a[0] * b[2] + a[2] * b[1];
        reall_t p = c1 - c2 * c2 / 3.0L, q = 2.0L * c2 * c2 * c2 / 27.0L - c2 * c1 / 3.0L + c0;
        reall_t rr = sqrtl(-p / 3.0L);
        reall_t arg = 3.0L * q / (2.0L * p * rr);
        if (arg > 1.0L) arg = 1.0L;
        if (arg < -1.0L) arg = -1.0L;
        reall_t th = acosl(arg) / 3.0L;
        const long double PI_L = 3.141592653589793238462643383279502884L;
        for (int i = 0; i < 3; i++) x[i] = 2.0L * rr * cosl(th - 2.0L * PI_L * i / 3.0L) - c2 / 3.0L;
        for (int i = 0; i < 3; i++)
            for (int it = 0; it < 2; it++) {
                reall_t v = ((x[i] + c2) * x[i] + c1) * x[i] + c0;
                reall_t dv = (3.0L * x[i] + 2.0L * c2) * x[i] + c1;
                if (dv != 0.0L) x[i] -= v / dv;
            }
        for (int i = 0; i < 3; i++)
            for (int j = i + 1; j < 3; j++)
                if (x[j] < x[i]) { reall_t t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (int i = 0; i < n; i++) {
        /* Christoffel number: b0 / sum_k p_k(x)^2 / (b1..bk), monic p_k */
        reall_t p0 = 1.0L, p1 = 0.0L, nrm = 1.0L, sm = 1.0L;
        for (int k = 0; k + 1 < n; k++) {
            reall_t pn = (x[i] - a[k]) * p0 - (k > 0 ? b[k] * p1 : (reall_t)0.0L);
            p1 = p0;
            p0 = pn;
            nrm *= b[k + 1];
            sm += p0 * p0 / nrm;
        }
        u[i] = (real_t)x[i];
        w[i] = (real_t)(b[0] / sm);
    }
}

/* Golub-Welsch step of the Rys classes (the reference's RYSGW): eigenvalues
 * of the symmetric tridiagonal Jacobi matrix (diagonal a[0..n-1], squared
 * off-diagonals b2[1..n-1]) by implicit QL iterations with Wilkinson shifts
 * (Golub and Welsch, Math. Comp. 23 (1969) 221), carrying the first row of
 * the eigenvector matrix, whose squares times the total mass beta0 are the
 * weights.  Roots ascending. */
static void rys_gw(int n, const real_t *a, const real_t *b2, real_t beta0, real_t *x, real_t *w) {
    real_t d[MAXROOT], e[MAXROOT], z[MAXROOT];
    for (int i = 0; i < n; i++) {
        d[i] = a[i];
        e[i] = i + 1 < n ? sqrt(b2[i + 1]) : (real_t)0.0;
        z[i] = i == 0 ? 1.0 : 0.0;
    }
    for (int l = 0; l < n; l++) {
        for (int iter = 0; iter < 60; iter++) {
            int m = l;
            while (m < n - 1 && !(fabs(e[m]) <= 1e-17 * (fabs(d[m]) + fabs(d[m + 1])))) m++;
            if (m == l) break;
            /* Wilkinson shift from the leading 2x2 block, then a chase of
             * plane rotations from row m-1 up to row l */
            real_t g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            real_t r = sqrt(g * g + 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            real_t sn = 1.0, cs = 1.0, p = 0.0;
            int i = m - 1;
            for (; i >= l; i--) {
                real_t f = sn * e[i], bb = cs * e[i];
                r = sqrt(f * f + g * g);
                e[i + 1] = r;
                if (r == 0.0) {  /* exact deflation */
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    break;
                }
                sn = f / r;
                cs = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * sn + 2.0 * cs * bb;
                p = sn * r;
                d[i + 1] = g + p;
                g = cs * r - bb;
                const real_t zt = z[i + 1];
                z[i + 1] = sn * z[i] + cs * zt;
                z[i] = cs * z[i] - sn * zt;
            }
            if (i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    for (int i = 0; i < n; i++) { x[i] = d[i]; w[i] = beta0 * z[i] * z[i]; }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (x[j] < x[i]) {
                real_t t = x[i]; x[i] = x[j]; x[j] = t;
                t = w[i]; w[i] = w[j]; w[j] = t;
            }
}

static void init_tables(void) {
    if (g_init) return;
    boys_table_init();
    for (int gs = 0; gs < 3; gs++) {
        const int ng = 30 + 5 * gs;
        double gx[MAXGRID], gw[MAXGRID];
        gauss_legendre(ng, gx, gw);
        for (int i = 0; i < ng; i++) {
            double t = 0.5 * (gx[i] + 1.0);
            GRID_U[gs][i] = t * t;
            GRID_W[gs][i] = 0.5 * gw[i];
        }
    }
    for (int n = 1; n <= MAXROOT; n++) {
        int m = 2 * n;
        double a[2 * MAXROOT], b2[2 * MAXROOT], x[2 * MAXROOT], w[2 * MAXROOT];
        for (int i = 0; i < m; i++) { a[i] = 0.0; b2[i] = 0.5 * i; }
        jacobi_gauss(m, a, b2, sqrt(PI_D), -(double)m, (double)m, x, w);
        for (int i = 0; i < n; i++) {
            HR[n][i] = x[n + i] * x[n + i];
            HW[n][i] = w[n + i];
        }
    }
    for (int l = 0; l <= MAXL; l++)
        for (int c = 0; c < MAXCART; c++) CNORM[l][c] = 1.0;
    CNORM[2][3] = CNORM[2][4] = CNORM[2][5] = sqrt(3.0);
    for (int c = 3; c < 9; c++) CNORM[3][c] = sqrt(5.0);
    CNORM[3][9] = sqrt(5.0) * sqrt(3.0);
    g_init = 1;
}

/* Rys roots u_i = t_i^2 in (0,1) and weights w_i (sum w_i = F_0(T)).
 * rot: 1 -> Boys-function rule, asymptotic when T > thr (rotated-axis and
 * ERIC kernels), 0 -> RYSDS on an ngrid-point grid, asymptotic for T >= thr */
static void rys_roots(int n, real_t T, double thr, int rot, int ngrid, real_t *u, real_t *w) {
    int asym = rot ? (T > thr) : (T >= thr);
    if (asym) {
        real_t it = 1.0 / T, sq = sqrt(it);
        for (int i = 0; i < n; i++) { u[i] = HR[n][i] * it; w[i] = HW[n][i] * sq; }
        return;
    }
    if (rot && n <= 2) {  /* rotated-axis classes: Boys-function moments */
        rys_small_d(n, T, u, w);
        return;
    }
    if (rot && n == 3) {
        rys_from_moments(n, T, u, w);
        return;
    }
    /* RYSDS: Stieltjes on the discrete measure {GRID_U, GRID_W*exp(-T u)} */
    const int NGRID = ngrid, gs = grid_slot(ngrid);
    const double *GU = GRID_U[gs], *GW = GRID_W[gs];
    real_t W[MAXGRID], p0[MAXGRID], p1[MAXGRID];
    real_t a[MAXROOT], b2[MAXROOT];
    real_t s0 = 0.0, s1 = 0.0;
    for (int j = 0; j < NGRID; j++) {
        W[j] = GW[j] * exp(-T * GU[j]);
        p0[j] = 1.0;
        p1[j] = 0.0;
        s0 += W[j];
        s1 += W[j] * GU[j];
    }
    real_t beta0 = s0, nprev = s0;
    a[0] = s1 / s0;
    b2[0] = 0.0;
    for (int k = 1; k < n; k++) {
        real_t sa = 0.0, sb = 0.0;
        for (int j = 0; j < NGRID; j++) {
            real_t pn = (GU[j] - a[k - 1]) * p0[j];
            if (k > 1) pn -= b2[k - 1] * p1[j];
            p1[j] = p0[j];
            p0[j] = pn;
            sa += W[j] * pn * pn;
            sb += W[j] * GU[j] * pn * pn;
        }
        a[k] = sb / sa;
        b2[k] = sa / nprev;
        nprev = sa;
    }
    rys_gw(n, a, b2, beta0, u, w);  /* RYSGW */
}

/* ============================ setup ========================================= */
static void free_ctx(ctx_t *c) {
    free(c->csh);
    for (int l = 0; l <= MAXL; l++) free(c->lst[l]);
    for (int k = 0; k < NPC; k++) {
        pairs_t *p = &c->pc[k];
        free(p->ish); free(p->jsh); free(p->xint); free(p->loc);
        free(p->ea); free(p->eb); free(p->cc); free(p->ismlp);
    }
}

static int64_t tri_idx(int64_t i, int64_t j) { /* 1-based ia(max)+min */
    if (i < j) { int64_t t = i; i = j; j = t; }
    return i * (i - 1) / 2 + j;
}

static void build_ctx(ctx_t *c, const oracle_basis *b) {
    memset(c, 0, sizeof(*c));
    c->b = b;
    c->coef[0] = b->coef_s; c->coef[1] = b->coef_p; c->coef[2] = b->coef_d; c->coef[3] = b->coef_f;
    c->csh = (double(*)[3])malloc(sizeof(double[3]) * (b->nsh > 0 ? b->nsh : 1));
    for (int s = 0; s < b->nsh; s++)
        for (int x = 0; x < 3; x++) c->csh[s][x] = b->coords[3 * (b->atom_num[s] - 1) + x];
    /* ascending per-L lists (classify_shells final sort, :301-344) */
    for (int l = 0; l <= MAXL; l++) {
        c->lst[l] = (int32_t *)malloc(sizeof(int32_t) * (b->nsh > 0 ? b->nsh : 1));
        c->nl[l] = 0;
    }
    for (int s = 0; s < b->nsh; s++) {
        int l = b->ang_mom[s] - 1;
        if (l >= 0 && l <= MAXL) c->lst[l][c->nl[l]++] = s;
    }
    for (int k = 0; k < NPC; k++) {
        int l1 = PC_L1[k], l2 = PC_L2[k];
        int same = (l1 == l2);
        int64_t n1 = c->nl[l1], n2 = c->nl[l2];
        pairs_t *p = &c->pc[k];
        p->n = same ? n1 * (n1 + 1) / 2 : n1 * n2;
        int64_t nn = p->n > 0 ? p->n : 1;
        p->ish = (int32_t *)malloc(sizeof(int32_t) * nn);
        p->jsh = (int32_t *)malloc(sizeof(int32_t) * nn);
        p->xint = (double *)malloc(sizeof(double) * nn);
        p->loc = (int64_t *)malloc(sizeof(int64_t) * (nn + 1));
        int64_t q = 0;
        p->loc[0] = 0;
        for (int64_t ii = 0; ii < n1; ii++) {
            int64_t jmax = same ? ii + 1 : n2;
            for (int64_t jj = 0; jj < jmax; jj++) {
                int32_t is = c->lst[l1][ii], js = c->lst[l2][jj];
                p->ish[q] = is;
                p->jsh[q] = js;
                p->xint[q] = b->schwrz[tri_idx(is + 1, js + 1) - 1];
                p->loc[q + 1] = p->loc[q] + (int64_t)b->contr_num[is] * b->contr_num[js];
                q++;
            }
        }
        int64_t np = p->loc[p->n];
        int64_t npp = np > 0 ? np : 1;
        p->ea = (double *)malloc(sizeof(double) * npp);
        p->eb = (double *)malloc(sizeof(double) * npp);
        p->cc = (double *)malloc(sizeof(double) * npp);
        p->ismlp = (int32_t *)malloc(sizeof(int32_t) * npp);
        for (int64_t e = 0; e < p->n; e++) {
            int is = p->ish[e], js = p->jsh[e];
            double r2 = 0.0;
            for (int x = 0; x < 3; x++) {
                double d = c->csh[js][x] - c->csh[is][x];
                r2 += d * d;
            }
            int64_t o = p->loc[e];
            for (int i = 0; i < b->contr_num[is]; i++) {
                double a = b->exponents[b->sh_loc[is] - 1 + i];
                double ca = c->coef[l1][b->sh_loc[is] - 1 + i];
                for (int j = 0; j < b->contr_num[js]; j++) {
                    double bb = b->exponents[b->sh_loc[js] - 1 + j];
                    double cb = c->coef[l2][b->sh_loc[js] - 1 + j];
                    double pinv = 1.0 / (a + bb);
                    double mur2 = r2 * (a * pinv) * bb;
                    p->ea[o] = a;
                    p->eb[o] = bb;
                    p->cc[o] = ca * cb;
                    p->ismlp[o] = (mur2 > CUX) ? 2 : 0;
                    o++;
                }
            }
        }
    }
}

/* ====================== shell-quartet integrals ============================= */
/* out[((i*nb + j)*nc + k)*nd + l] contracted Cartesian integrals */
static int64_t eri_quartet(const ctx_t *c, int A, int B, int C, int D,
                           const pairs_t *pb, int64_t eb_, const pairs_t *pk, int64_t ek_,
                           const kdesc_t *kd, real_t *out) {
    const oracle_basis *b = c->b;
    /* out keeps the (A B|C D) order of the call; the evaluation puts the
     * higher-L shell of each pair first, as the reference's Rys kernels order
     * their pairs (int3011_rysgen.F90: ish the f shell of an sf pair): the
     * transfer relation then moves angular momentum onto the lower-L shell,
     * which stays accurate when a tight high-L shell meets a distant diffuse
     * partner (the other way round loses digits to cancellation) */
    const int la0 = b->ang_mom[A] - 1, lb0 = b->ang_mom[B] - 1, lc0 = b->ang_mom[C] - 1, ld0 = b->ang_mom[D] - 1;
    const int nb0 = NCART[lb0], nc0 = NCART[lc0], nd0 = NCART[ld0];
    const int sab = lb0 > la0, scd = ld0 > lc0;
    if (sab) { const int t = A; A = B; B = t; }
    if (scd) { const int t = C; C = D; D = t; }
    int la = b->ang_mom[A] - 1, lb = b->ang_mom[B] - 1, lc = b->ang_mom[C] - 1, ld = b->ang_mom[D] - 1;
    int na = NCART[la], nb = NCART[lb], nc = NCART[lc], nd = NCART[ld];
    int n = (la + lb + lc + ld) / 2 + 1;
    int nij = la + lb, nkl = lc + ld;
    const double *Ar = c->csh[A], *Br = c->csh[B], *Cr = c->csh[C], *Dr = c->csh[D];
    real_t AB[3], CD[3], rab2 = 0.0, rcd2 = 0.0;
    for (int x = 0; x < 3; x++) {
        AB[x] = Ar[x] - Br[x]; CD[x] = Cr[x] - Dr[x];
        rab2 += AB[x] * AB[x]; rcd2 += CD[x] * CD[x];
    }
    int ntot = na * nb * nc * nd;
    for (int i = 0; i < ntot; i++) out[i] = 0.0;
    int64_t nprim = 0;
    const double twopi52 = 2.0 * PI_D * PI_D * sqrt(PI_D);
    for (int64_t kq = pk->loc[ek_]; kq < pk->loc[ek_ + 1]; kq++) {
        real_t gc = scd ? pk->eb[kq] : pk->ea[kq], gd = scd ? pk->ea[kq] : pk->eb[kq], q = gc + gd;
        real_t Q[3];
        for (int x = 0; x < 3; x++) Q[x] = (gc * Cr[x] + gd * Dr[x]) / q;
        real_t ecd = exp(-gc * gd / q * rcd2);
        for (int64_t bq = pb->loc[eb_]; bq < pb->loc[eb_ + 1]; bq++) {
            if (kd->skip && (pb->ismlp[bq] + pk->ismlp[kq] >= 2)) continue;
            real_t ga = sab ? pb->eb[bq] : pb->ea[bq], gb = sab ? pb->ea[bq] : pb->eb[bq], p = ga + gb;
            real_t P[3], PQ2 = 0.0;
            for (int x = 0; x < 3; x++) {
                P[x] = (ga * Ar[x] + gb * Br[x]) / p;
                PQ2 += (P[x] - Q[x]) * (P[x] - Q[x]);
            }
            real_t eab = exp(-ga * gb / p * rab2);
            real_t rho = p * q / (p + q);
            real_t T = rho * PQ2;
            real_t u[MAXROOT], w[MAXROOT];
            rys_roots(n, T, kd->asym, !kd->rys, kd->ngrid, u, w);
            real_t pref = twopi52 * (pb->cc[bq] / p) * (pk->cc[kq] / q) * eab * ecd / sqrt(p + q);
            nprim++;
            /* 2D integrals per root and dimension: vertical recurrence, then
             * horizontal transfer to I[a][b][c][d] by recurrences */
            real_t I2[MAXROOT][3][MAXL + 1][MAXL + 1][MAXL + 1][MAXL + 1];
            const real_t ipq = 1.0 / (p + q);
            for (int r = 0; r < n; r++) {
                real_t ur = u[r];
                real_t B00 = 0.5 * ur * ipq;
                real_t B10 = 0.5 / p * (1.0 - q * ur * ipq);
                real_t B01 = 0.5 / q * (1.0 - p * ur * ipq);
                for (int x = 0; x < 3; x++) {
                    real_t C00 = (P[x] - Ar[x]) - q * ur * ipq * (P[x] - Q[x]);
                    real_t Cp00 = (Q[x] - Cr[x]) + p * ur * ipq * (P[x] - Q[x]);
                    real_t g[2 * MAXL + 1][2 * MAXL + 1];
                    g[0][0] = 1.0;
                    for (int i = 0; i < nij; i++) {
                        g[i + 1][0] = C00 * g[i][0];
                        if (i > 0) g[i + 1][0] += (double)i * B10 * g[i - 1][0];
                    }
                    for (int k = 0; k < nkl; k++) {
                        for (int i = 0; i <= nij; i++) {
                            real_t v = Cp00 * g[i][k];
                            if (k > 0) v += (double)k * B01 * g[i][k - 1];
                            if (i > 0) v += (double)i * B00 * g[i - 1][k];
                            g[i][k + 1] = v;
                        }
                    }
                    real_t h[2 * MAXL + 1][MAXL + 1][2 * MAXL + 1];
                    for (int e = 0; e <= nij; e++)
                        for (int f = 0; f <= nkl; f++) h[e][0][f] = g[e][f];
                    for (int bb = 1; bb <= lb; bb++)
                        for (int a2 = 0; a2 <= nij - bb; a2++)
                            for (int f = 0; f <= nkl; f++) h[a2][bb][f] = h[a2 + 1][bb - 1][f] + AB[x] * h[a2][bb - 1][f];
                    for (int a2 = 0; a2 <= la; a2++)
                        for (int bb = 0; bb <= lb; bb++) {
                            real_t k2[2 * MAXL + 1][MAXL + 1];
                            for (int f = 0; f <= nkl; f++) k2[f][0] = h[a2][bb][f];
                            for (int dd = 1; dd <= ld; dd++)
                                for (int cc = 0; cc <= nkl - dd; cc++) k2[cc][dd] = k2[cc + 1][dd - 1] + CD[x] * k2[cc][dd - 1];
                            for (int cc = 0; cc <= lc; cc++)
                                for (int dd = 0; dd <= ld; dd++) I2[r][x][a2][bb][cc][dd] = k2[cc][dd];
                        }
                }
            }
            /* assembly */
            for (int ia = 0; ia < na; ia++)
            for (int ib = 0; ib < nb; ib++)
            for (int ic = 0; ic < nc; ic++)
            for (int id = 0; id < nd; id++) {
                const int ax = CX[la][ia], ay = CY[la][ia], az = CZ[la][ia];
                const int bx = CX[lb][ib], by = CY[lb][ib], bz = CZ[lb][ib];
                const int cx = CX[lc][ic], cy = CY[lc][ic], cz = CZ[lc][ic];
                const int dx = CX[ld][id], dy = CY[ld][id], dz = CZ[ld][id];
                real_t acc = 0.0;
                for (int r = 0; r < n; r++)
                    acc += w[r] * I2[r][0][ax][bx][cx][dx] * I2[r][1][ay][by][cy][dy] * I2[r][2][az][bz][cz][dz];
                const int i0 = sab ? ib : ia, j0 = sab ? ia : ib, k0 = scd ? id : ic, l0 = scd ? ic : id;
                out[((i0 * nb0 + j0) * nc0 + k0) * nd0 + l0] += pref * acc;
            }
        }
    }
    ORACLE_MARK();  /* op-counting build: end of the primitive-quartet work */
    /* component normalisation (sqrt3 on xy,xz,yz of d; sqrt5 / sqrt15 on f),
     * in the call's order */
    for (int ia = 0; ia < NCART[la0]; ia++)
    for (int ib = 0; ib < nb0; ib++)
    for (int ic = 0; ic < nc0; ic++)
    for (int id = 0; id < nd0; id++)
        out[((ia * nb0 + ib) * nc0 + ic) * nd0 + id] *=
            CNORM[la0][ia] * CNORM[lb0][ib] * CNORM[lc0][ic] * CNORM[ld0][id];
    return nprim;
}

/* =============================== DIRFCK ===================================== */
/* Dm: the density of the Coulomb updates (F(ij) += 4 v D(kl)); Dk: that of the
 * exchange updates (F(ik) -= v D(jl) ...), Dm itself for a closed-shell build */
static int64_t dirfck(const ctx_t *c, int A, int B, int C, int D, const real_t *v,
                      double cut, const double *Dm, const double *Dk, double *F) {
    const oracle_basis *b = c->b;
    int na = NCART[b->ang_mom[A] - 1], nb = NCART[b->ang_mom[B] - 1];
    int nc = NCART[b->ang_mom[C] - 1], nd = NCART[b->ang_mom[D] - 1];
    int iandj = (A == B), kandl = (C == D), same = (A == C && B == D);
    int64_t loci = b->atom_loc[A] - 1, locj = b->atom_loc[B] - 1;
    int64_t lock = b->atom_loc[C] - 1, locl = b->atom_loc[D] - 1;
    int64_t ndig = 0;
    int nij = 0;
    for (int i = 0; i < na; i++) {
        int maxj2 = iandj ? i + 1 : nb;
        for (int j = 0; j < maxj2; j++) {
            nij++;
            int nkl = nij;
            int maxl2 = nd;
            for (int k = 0; k < nc; k++) {
                if (kandl) maxl2 = k + 1;
                if (same) {
                    int itmp = maxl2 < nkl ? maxl2 : nkl;
                    if (itmp == 0) break;
                    maxl2 = itmp;
                    nkl -= itmp;
                }
                for (int l = 0; l < maxl2; l++) {
                    real_t val = v[((i * nb + j) * nc + k) * nd + l];
                    if (fabs(val) < cut) continue;
                    ndig++;
                    int64_t i1 = i + 1 + loci, j1 = j + 1 + locj, k1 = k + 1 + lock, l1 = l + 1 + locl;
                    int64_t i2 = i1, j2 = j1, k2 = k1, l2 = l1;
                    if (i1 < j1) { i2 = j1; j2 = i1; }
                    if (k1 < l1) { k2 = l1; l2 = k1; }
                    int64_t ii = i2, jj = j2, kk = k2, ll = l2;
                    if (ii < kk) { ii = k2; jj = l2; kk = i2; ll = j2; }
                    else if (ii == kk && jj < ll) { jj = l2; ll = j2; }
                    int64_t ij = tri_idx(ii, jj), ik = tri_idx(ii, kk), il = tri_idx(ii, ll);
                    int64_t jk = tri_idx(jj, kk), jl = tri_idx(jj, ll), kl = tri_idx(kk, ll);
                    if (ii == jj) val *= 0.5;
                    if (kk == ll) val *= 0.5;
                    if (ii == kk && jj == ll) val *= 0.5;
                    real_t v4 = 4.0 * val;
                    F[ij - 1] = (double)(F[ij - 1] + v4 * Dm[kl - 1]);
                    F[kl - 1] = (double)(F[kl - 1] + v4 * Dm[ij - 1]);
                    F[ik - 1] = (double)(F[ik - 1] - val * Dk[jl - 1]);
                    F[jl - 1] = (double)(F[jl - 1] - val * Dk[ik - 1]);
                    F[il - 1] = (double)(F[il - 1] - val * Dk[jk - 1]);
                    F[jk - 1] = (double)(F[jk - 1] - val * Dk[il - 1]);
                }
            }
        }
    }
    return ndig;
}

/* ======================= screening and rank split ========================== */
static double maxval(const pairs_t *p) {
    double m = -HUGE_VAL;
    for (int64_t i = 0; i < p->n; i++) if (p->xint[i] > m) m = p->xint[i];
    return m;
}

/* does 1-based iteration index `it` of a kernel with `ntot` iterations belong
 * to rank my_rank?  Mirrors the tile + rank arithmetic of each kernel, e.g.
 * int0000.F90:76-91, int0001.F90:89-104, int0101.F90:76-79 */
int oracle_rank_owns(int tile, int64_t ntot, int64_t it, int rank, int nsize) {
    if (ntot <= 0) return 0;
    if (tile == TILE_NONE) {
        int64_t nchunk = ntot / nsize;
        int64_t s = nchunk * rank + 1, e = s + nchunk - 1;
        if (rank == nsize - 1) e = ntot;
        return it >= s && it <= e;
    }
    int64_t chunk;
    if (tile == TILE_SQRT) chunk = (int64_t)sqrt(375000000.0 * 10.0);
    else if (tile == TILE_E9) chunk = (int64_t)(375000000.0 * 10.0);
    else chunk = 375000000;
    if (ntot <= chunk) chunk = ntot;
    int64_t ntile = ntot / chunk;
    int64_t t = (it - 1) / chunk + 1;
    if (t > ntile) t = ntile;
    int64_t is = (t - 1) * chunk + 1, ie = t * chunk;
    if (t == ntile) ie = ntot;
    int64_t nchunk = (ie - is) / nsize;
    int64_t s = nchunk * rank + is, e = s + nchunk - 1;
    if (rank == nsize - 1) e = ie;
    return it >= s && it <= e;
}

static double now_s(void) {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

static uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

/* 64-bit fingerprint of one shell quartet, independent of the orientation of
 * each pair and of bra/ket order: shells (0-based, < 65536) form unordered
 * pair keys, the two pair keys an unordered quartet key, mixed by mix64 */
static uint64_t quartet_fp(int A, int B, int C, int D) {
    uint64_t p1 = A > B ? ((uint64_t)A << 16 | (uint64_t)B) : ((uint64_t)B << 16 | (uint64_t)A);
    uint64_t p2 = C > D ? ((uint64_t)C << 16 | (uint64_t)D) : ((uint64_t)D << 16 | (uint64_t)C);
    return mix64(p1 > p2 ? (p1 << 32 | p2) : (p2 << 32 | p1));
}

/* ============================== driver ====================================== */
int oracle_fock_build_jk(const oracle_basis *b, const oracle_opts *o, const double *Dm, const double *Dk,
                         double *F, oracle_counts *cnt);

/* Closed-shell build (liberi_fock_build): one density for every update. */
int oracle_fock_build(const oracle_basis *b, const oracle_opts *o, const double *Dm,
                      double *F, oracle_counts *cnt) {
    return oracle_fock_build_jk(b, o, Dm, Dm, F, cnt);
}

/* Build with separate Coulomb (Dm) and exchange (Dk) densities: the open-shell
 * form F_spin = J(D_alpha + D_beta) - K(2 D_spin) is Dm = D_alpha + D_beta,
 * Dk = 2 D_spin (libERI itself is closed-shell only). */
int oracle_fock_build_jk(const oracle_basis *b, const oracle_opts *o, const double *Dm, const double *Dk,
                         double *F, oracle_counts *cnt) {
    init_tables();
    int64_t nbf = b->num_bas, ntri = nbf * (nbf + 1) / 2;
    for (int64_t i = 0; i < ntri; i++) F[i] = 0.0; /* liberi_driver.F90:64 */
    if (cnt) memset(cnt, 0, sizeof(*cnt));
    ctx_t c;
    build_ctx(&c, b);
    int nth = 1;
#ifdef _OPENMP
    nth = o->nthreads > 0 ? o->nthreads : omp_get_max_threads();
#endif
    double *Fp = (double *)calloc((size_t)nth * ntri, sizeof(double));
    for (int kk = 0; kk < NK; kk++) {
        const kdesc_t *kd = &KD[kk];
        if (o->only_kernel >= 0 && o->only_kernel != kk) continue;
        /* driver guards (liberi_driver.F90:69-81) */
        if (kk == 0 && c.nl[0] == 0) continue;
        if (kk >= 1 && kk <= 5 && c.nl[1] == 0) continue;
        if (kk >= 6 && kk < 21 && c.nl[2] == 0) continue;
        if (kk >= 21 && c.nl[3] == 0) continue;  /* ENABLE_F block (liberi_driver.F90:103-160) */
        const pairs_t *pb = &c.pc[kd->bra], *pk = &c.pc[kd->ket];
        if (pb->n == 0 || pk->n == 0) continue;
        /* pre-screen: cross-class maxima for rotated-axis mixed kernels,
         * own-class maxima for same-class and Rys kernels */
        double sb = o->schwarz_cut / maxval(kd->cross ? pk : pb);
        double sk = o->schwarz_cut / maxval(kd->cross ? pb : pk);
        int64_t *lb = (int64_t *)malloc(sizeof(int64_t) * pb->n), *lk = (int64_t *)malloc(sizeof(int64_t) * pk->n);
        int64_t nbl = 0, nkl = 0;
        for (int64_t i = 0; i < pb->n; i++) if (pb->xint[i] >= sb) lb[nbl++] = i;
        if (kd->tri) { memcpy(lk, lb, sizeof(int64_t) * nbl); nkl = nbl; }
        else for (int64_t i = 0; i < pk->n; i++) if (pk->xint[i] >= sk) lk[nkl++] = i;
        if (nbl == 0 || nkl == 0) { free(lb); free(lk); continue; }
        double dcut = kd->digest_schwarz ? o->schwarz_cut : o->eri_cut;
        int64_t niter = kd->tri ? nbl : nbl * nkl;
        int64_t c_scr = 0, c_prim = 0, c_dig = 0, c_eval = 0;
        uint64_t fp_sum = 0, fp_xor = 0, ops_prim = 0, ops_shell = 0;
        double t_eval = 0.0, t_k0 = now_s();
#pragma omp parallel num_threads(nth) reduction(+ : c_scr, c_prim, c_dig, c_eval, t_eval, fp_sum, ops_prim, ops_shell) reduction(^ : fp_xor)
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double *Ft = Fp + (size_t)tid * ntri;
            real_t vbuf[MAXCART * MAXCART * MAXCART * MAXCART];
#pragma omp for schedule(dynamic, 16)
            for (int64_t it = 1; it <= niter; it++) {
                if (o->num_procs > 1 && !oracle_rank_owns(kd->tile, niter, it, o->my_rank, o->num_procs)) continue;
                int64_t jb_lo, jb_hi, ib;
                if (kd->tri) { ib = it - 1; jb_lo = 0; jb_hi = it; }
                else { jb_lo = 0; jb_hi = 1; ib = 0; }
                for (int64_t jq = jb_lo; jq < jb_hi; jq++) {
                    int64_t bi, ki;
                    if (kd->tri) { bi = lb[ib]; ki = lb[jq]; }
                    else if (kd->ketmajor) { bi = lb[(it - 1) % nbl]; ki = lk[(it - 1) / nbl]; }
                    else { bi = lb[(it - 1) / nkl]; ki = lk[(it - 1) % nkl]; }
                    double test = pb->xint[bi] * pk->xint[ki];
                    if (kd->op == OP_GE && !(test >= o->schwarz_cut)) continue;
                    if (kd->op == OP_GT && !(test > o->schwarz_cut)) continue;
                    c_scr++;
                    {
                        const uint64_t f = quartet_fp(pb->ish[bi], pb->jsh[bi], pk->ish[ki], pk->jsh[ki]);
                        fp_sum += f;
                        fp_xor ^= f;
                    }
                    if (o->sample_mod > 1) {
                        /* sample whole bra pairs (all their kets), so the sampled
                         * work keeps the cache behaviour of a full run */
                        uint64_t h = mix64(((uint64_t)kk << 56) ^ ((uint64_t)bi << 8) ^ ((uint64_t)o->sample_seed << 40));
                        if (h % (uint64_t)o->sample_mod) continue;
                    }
                    c_eval++;
                    double tq = o->sample_mod > 1 ? now_s() : 0.0;
                    int A = pb->ish[bi], B = pb->jsh[bi], C = pk->ish[ki], D = pk->jsh[ki];
                    const uint64_t o0 = ORACLE_OPS();
                    c_prim += eri_quartet(&c, A, B, C, D, pb, bi, pk, ki, kd, vbuf);
                    const uint64_t o1 = ORACLE_OPS();
                    c_dig += dirfck(&c, A, B, C, D, vbuf, dcut, Dm, Dk, Ft);
                    /* primitive work up to eri_quartet's mark; its normalisation
                     * and the digestion are shell-quartet work */
                    ops_prim += ORACLE_MARKED() - o0;
                    ops_shell += (o1 - ORACLE_MARKED()) + (ORACLE_OPS() - o1);
                    if (o->sample_mod > 1) t_eval += now_s() - tq;
                }
            }
        }
        if (cnt) {
            cnt->c[kk][0] = c_scr; cnt->c[kk][1] = c_prim;
            cnt->c[kk][2] = c_dig; cnt->c[kk][3] = c_eval;
            cnt->t_wall[kk] = now_s() - t_k0;
            cnt->t_eval[kk] = t_eval;
            cnt->nthreads = nth;
            cnt->fp[kk][0] = fp_sum;
            cnt->fp[kk][1] = fp_xor;
            cnt->ops[kk][0] = ops_prim;
            cnt->ops[kk][1] = ops_shell;
        }
        free(lb); free(lk);
    }
    for (int t = 0; t < nth; t++)
        for (int64_t i = 0; i < ntri; i++) F[i] += Fp[(size_t)t * ntri + i];
    free(Fp);
    free_ctx(&c);
    return 0;
}

/* Schwarz table Q_ab = sqrt(max_component |(ab|ab)|), packed over shells with
 * ia(max)+min.  The reference receives this table from GAMESS
 * (liberi_interface.F90:128-129); the oracle provides it for synthetic inputs. */
int oracle_schwarz(const oracle_basis *b, double *schwrz_out) {
    init_tables();
    /* evaluate with a Rys-style descriptor: no primitive skipping, the
     * 40-point procedure below T = 60 and the large-T form above it (the
     * 40-point grid integrates the moments of up to 7 roots to ~1e-15 there) */
    kdesc_t kd = {"schwarz", 0, 0, 0, 1, 0, OP_NONE, TILE_NONE, 0, 0, 60.0, 40, 0};
    oracle_basis bb = *b;
    int64_t ntri = (int64_t)b->nsh * (b->nsh + 1) / 2;
    double *dummy = (double *)malloc(sizeof(double) * (ntri > 0 ? ntri : 1));
    for (int64_t i = 0; i < ntri; i++) dummy[i] = 1.0;
    bb.schwrz = dummy;
    ctx_t c;
    build_ctx(&c, &bb);
    for (int64_t i = 0; i < ntri; i++) schwrz_out[i] = 0.0;
    for (int k = 0; k < NPC; k++) {
        const pairs_t *p = &c.pc[k];
#pragma omp parallel for schedule(dynamic, 4)
        for (int64_t e = 0; e < p->n; e++) {
            real_t v[MAXCART * MAXCART * MAXCART * MAXCART];
            int A = p->ish[e], B = p->jsh[e];
            eri_quartet(&c, A, B, A, B, p, e, p, e, &kd, v);
            int na = NCART[b->ang_mom[A] - 1], nb = NCART[b->ang_mom[B] - 1];
            double m = 0.0;
            for (int i = 0; i < na; i++)
                for (int j = 0; j < nb; j++) {
                    double x = (double)fabs(v[((i * nb + j) * na + i) * nb + j]);
                    if (x > m) m = x;
                }
            schwrz_out[tri_idx(A + 1, B + 1) - 1] = sqrt(m);
        }
    }
    free_ctx(&c);
    free(dummy);
    return 0;
}

/* Exposes the Rys root routine for the table-accuracy tests: the grid of the
 * reference's kernels with n roots (30 points up to 4 roots, 35 for 5, 40 for
 * 6 and 7), or ngrid points. */
void oracle_rys_roots_grid(int n, double T, double thr, int rot, int ngrid, double *u, double *w) {
    init_tables();
    real_t ur[MAXROOT], wr[MAXROOT];
    if (n < 1 || n > MAXROOT) return;
    rys_roots(n, T, thr, rot, ngrid, ur, wr);
    for (int i = 0; i < n; i++) { u[i] = (double)ur[i]; w[i] = (double)wr[i]; }
}

void oracle_rys_roots(int n, double T, double thr, int rot, double *u, double *w) {
    oracle_rys_roots_grid(n, T, thr, rot, n <= 4 ? 30 : (n == 5 ? 35 : 40), u, w);
}

int oracle_num_kernels(void) { return NK; }
const char *oracle_kernel_name(int k) { return (k >= 0 && k < NK) ? KD[k].name : ""; }
