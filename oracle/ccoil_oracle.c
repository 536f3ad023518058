/*
 * ccoil_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, double-precision restatement of the reference's CPU algorithm for
 * the field and coil-pair hot path of C-Coil.  It is the checker for the CUDA
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it.  The product never links or calls it.
 *
 * Parity pin: tests/test_oracle.py checks every function here against the
 * reference itself (oracle/_ref/libccoil_ref.so, compiled from the reference's
 * own sources) and against the committed golden vectors in tests/golden/.
 *
 * Conventions (shared with the reference):
 *   coil parameters  {R, a, b, N, I, f, x, y, z, yAxisAngle, zAxisAngle}
 *   precision args   {angularBlocks, thicknessBlocks, lengthBlocks,
 *                     angularIncrements, thicknessIncrements, lengthIncrements}
 *   points           interleaved xyz
 * Gauss-Legendre nodes are computed here (Newton iteration on P_n) rather than
 * read from the reference's literal table; they agree with it to within 1 ulp.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAX_ORDER 100
#define MI_REDUCED 1e-7
#define THIN_RATIO 1e-7          /* g_thinCoilApproximationRatio, PrecisionGlobalVars.h:18 */
#define ZAXIS_RATIO 1e-12        /* g_zAxisApproximationRatio, PrecisionGlobalVars.h:19 */
#define PLANE_RATIO 1e-14        /* g_commonPlaneApproximationRatio, PrecisionGlobalVars.h:20 */
#define PRIM_MOD 1.414213562     /* g_prim{Angular,Linear}WeightModifier, PrecisionGlobalVars.h:12-13 */

static const double PI = 3.14159265358979323846;

/* ------------------------------------------------------------------ */
/* Gauss-Legendre nodes and weights                                    */
/* ------------------------------------------------------------------ */
static double g_pos[MAX_ORDER][MAX_ORDER];
static double g_wts[MAX_ORDER][MAX_ORDER];
static int g_ready = 0;

static void legendre_eval(int n, long double x, long double *p, long double *dp)
{
    long double p0 = 1.0L, p1 = x;
    if (n == 0) { *p = 1.0L; *dp = 0.0L; return; }
    for (int k = 2; k <= n; ++k)
    {
        long double pk = ((2.0L * k - 1.0L) * x * p1 - (k - 1.0L) * p0) / k;
        p0 = p1;
        p1 = pk;
    }
    *p = p1;
    *dp = n * (x * p1 - p0) / (x * x - 1.0L);
}

static void build_tables(void)
{
    if (g_ready)
        return;
    for (int n = 1; n <= MAX_ORDER; ++n)
    {
        int half = n / 2;
        for (int i = 0; i < half; ++i)
        {
            /* i-th root from the largest down: cos(pi (i + 0.75) / (n + 0.5)) */
            long double x = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
            long double p, dp;
            for (int it = 0; it < 100; ++it)
            {
                legendre_eval(n, x, &p, &dp);
                long double dx = p / dp;
                x -= dx;
                if (fabsl(dx) < 1e-22L)
                    break;
            }
            legendre_eval(n, x, &p, &dp);
            long double w = 2.0L / ((1.0L - x * x) * dp * dp);
            /* ascending order: the positive root goes to the top, mirrored below */
            g_pos[n - 1][n - 1 - i] = (double)x;
            g_pos[n - 1][i] = -(double)x;
            g_wts[n - 1][n - 1 - i] = (double)w;
            g_wts[n - 1][i] = (double)w;
        }
        if (n % 2 == 1)
        {
            long double p, dp;
            legendre_eval(n, 0.0L, &p, &dp);
            g_pos[n - 1][half] = 0.0;
            g_wts[n - 1][half] = (double)(2.0L / (dp * dp));
        }
    }
    g_ready = 1;
}

int oracle_legendre(int order, double *pos, double *w)
{
    build_tables();
    if (order < 1 || order > MAX_ORDER)
        return -1;
    for (int i = 0; i < order; ++i)
    {
        pos[i] = g_pos[order - 1][i];
        w[i] = g_wts[order - 1][i];
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Coil attributes                                                      */
/* ------------------------------------------------------------------ */
enum { RECTANGULAR = 0, THIN = 1, FLAT = 2, FILAMENT = 3 };

typedef struct
{
    double R, a, b;        /* after the thin-dimension substitution */
    int N;
    double I, f, J;
    double pos[3];
    double yAngle, zAngle;
    double T[9], Tinv[9];
    int fast, type;
} OCoil;

/* Coil::Coil (src/Coil/Coil.cxx:22-44) with calculateCoilType and
 * calculateTransformationMatrices (src/Coil/Utils/CalculateAttributes.cxx:50-78) */
static void make_coil(const double *c, OCoil *k)
{
    double R = c[0], a = c[1], b = c[2];
    k->R = R;
    k->a = (a / R < THIN_RATIO) ? 1e-18 * R * THIN_RATIO : a;
    k->b = (b / R < THIN_RATIO) ? 1e-18 * R * THIN_RATIO : b;
    k->N = (int)c[3];
    k->fast = (b / R >= THIN_RATIO);
    k->I = c[4];
    k->f = c[5] > 0.0 ? c[5] : 0.0;
    k->J = k->I * k->N / (k->b * k->a);
    k->pos[0] = c[6]; k->pos[1] = c[7]; k->pos[2] = c[8];
    k->yAngle = c[9];
    k->zAngle = c[10];
    if (k->a / R < THIN_RATIO && k->b / R < THIN_RATIO) k->type = FILAMENT;
    else if (k->a / R < THIN_RATIO) k->type = THIN;
    else if (k->b / R < THIN_RATIO) k->type = FLAT;
    else k->type = RECTANGULAR;

    double cY = cos(k->yAngle), sY = sin(k->yAngle), cZ = cos(k->zAngle), sZ = sin(k->zAngle);
    double T[9] = {cZ * cZ * cY - sZ * sZ, -sZ * cZ * cY - sZ * cZ, cZ * sY,
                   sZ * cZ * cY + sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY,
                   -sY * cZ, sY * sZ, cY};
    double Ti[9] = {cZ * cZ * cY - sZ * sZ, sZ * cZ * cY + sZ * cZ, -cZ * sY,
                    -sZ * cZ * cY - sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY,
                    sY * cZ, sY * sZ, cY};
    memcpy(k->T, T, sizeof T);
    memcpy(k->Tinv, Ti, sizeof Ti);
}

int oracle_coil_info(const double *c, double *out)
{
    OCoil k;
    make_coil(c, &k);
    out[0] = k.a; out[1] = k.b; out[2] = k.J; out[3] = k.I;
    out[4] = k.fast; out[5] = k.type;
    memcpy(out + 6, k.T, sizeof k.T);
    memcpy(out + 15, k.Tinv, sizeof k.Tinv);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Precision arguments                                                  */
/* ------------------------------------------------------------------ */
typedef struct { int aB, tB, lB, aI, tI, lI; } OArgs;

/* PrecisionArguments ctor clamps (src/Coil/PrecisionArguments/PrecisionArguments.cxx:29-54) */
static OArgs make_args(int aB, int tB, int lB, int aI, int tI, int lI)
{
    OArgs r = {aB, tB, lB, aI, tI, lI};
    if (aI > MAX_ORDER || aI < 1) r.aI = 20;
    if (tI > MAX_ORDER || tI < 1) r.tI = 20;
    if (lI > MAX_ORDER || lI < 1) r.lI = 20;
    if (aB < 1) r.aB = 1;
    if (tB < 1) r.tB = 1;
    if (lI < 1) r.lB = 1;
    return r;
}

/* CoilPairArguments::balanceIncrements (src/Coil/PrecisionArguments/CoilPairArguments.cxx:20-46) */
static void balance(int total, int n, const double *meas, int *counts)
{
    if (n < 2)
    {
        counts[0] = total;
        return;
    }
    double eff = 1.0;
    for (int i = 0; i < n; ++i)
        eff *= meas[i];
    eff /= (double)total;
    double lin = pow(eff, 1.0 / (double)n);
    for (int i = 0; i < n; ++i)
        counts[i] = (int)round(meas[i] / lin);
}

/* the common split of one layer's increment count into Gauss-Legendre blocks
 * (PrecisionArguments.cxx:163-174, CoilPairArguments.cxx:222-233) */
static void split_blocks(int layer, int *blocks, int *incs)
{
    *blocks = (layer - 1) / MAX_ORDER + 1;
    *incs = (*blocks > 1) ? layer / *blocks + 1 : layer;
}

/* spill loop shared by the single-coil and pair balancing: a component whose
 * count exceeds the cap is pinned at the cap and removed, the total is reduced
 * and the rest is rebalanced */
static void balance_with_cap(int *total, int *ncomp, int *ids, double *meas, int *layer, int cap, const int *cappable)
{
    int counts[6];
    int spill;
    do
    {
        balance(*total, *ncomp, meas, counts);
        spill = 0;
        if (cap > 0)
        {
            for (int i = 0; i < *ncomp; ++i)
            {
                if (counts[i] > cap && (!cappable || cappable[ids[i]]))
                {
                    layer[ids[i]] = cap;
                    for (int j = i; j < *ncomp - 1; ++j)
                    {
                        ids[j] = ids[j + 1];
                        meas[j] = meas[j + 1];
                        counts[j] = counts[j + 1];
                    }
                    (*ncomp)--;
                    *total = (int)ceil((double)*total / (double)cap);
                    spill = 1;
                    break;
                }
            }
        }
    } while (spill && *ncomp > 0);
    for (int i = 0; i < *ncomp; ++i)
        layer[ids[i]] = counts[i];
}

/* PrecisionArguments::calculatePrecisionArguments (PrecisionArguments.cxx:69-185);
 * gpu_cap = 0 for the CPU variant, GPU_INCREMENTS for the GPU variant */
static OArgs coil_args(const OCoil *k, double pf, int gpu_cap)
{
    int layer[3] = {1, 1, 1};
    double measures[3];
    measures[0] = PRIM_MOD * sqrt(PI * (k->R + 0.5 * k->a));
    measures[1] = PRIM_MOD * sqrt(k->a);
    measures[2] = PRIM_MOD * sqrt(k->b);

    int ids[3], n = 0, total = 1;
    double meas[3];
    ids[n] = 0; meas[n++] = measures[0];
    total *= 10;
    if (k->type == RECTANGULAR || k->type == FLAT)
    {
        total *= 10;
        ids[n] = 1; meas[n++] = measures[1];
    }
    total = (int)((double)total * pow(2, pf - 1.0));
    balance_with_cap(&total, &n, ids, meas, layer, gpu_cap, NULL);

    if (layer[2] == 1)
        layer[2] = (int)round((double)layer[0] * measures[2] / measures[0]);
    if (layer[2] == 0)
        layer[2] = 1;
    if (gpu_cap > 0 && layer[2] > gpu_cap)
        layer[2] = gpu_cap;

    int b[3], inc[3];
    for (int i = 0; i < 3; ++i)
        split_blocks(layer[i], &b[i], &inc[i]);
    return make_args(b[0], b[1], b[2], inc[0], inc[1], inc[2]);
}

static double sanitize_pf(double pf) { return (pf < 1.0 || pf > 15.0) ? 5.0 : pf; }

int oracle_precision_args(const double *c, double pf, int gpu_cap, int *out6)
{
    OCoil k;
    make_coil(c, &k);
    OArgs a = coil_args(&k, sanitize_pf(pf), gpu_cap);
    int v[6] = {a.aB, a.tB, a.lB, a.aI, a.tI, a.lI};
    memcpy(out6, v, sizeof v);
    return 0;
}

/* CoilPairArguments::getAppropriateCoilPairArguments (CoilPairArguments.cxx:49-255) */
static void pair_args(const OCoil *p, const OCoil *s, double pf, int gpu_cap, int zAxis, int pureGPU,
                      OArgs *prim, OArgs *sec)
{
    int layer[6] = {1, 1, 1, 1, 1, 1};
    double measures[6];
    measures[0] = PRIM_MOD * sqrt(PI * (p->R + 0.5 * p->a));
    measures[1] = PRIM_MOD * sqrt(p->a);
    measures[2] = PRIM_MOD * sqrt(p->b);
    measures[3] = 1.0 * sqrt(2 * PI * (s->R + 0.5 * s->a));
    measures[4] = 1.0 * sqrt(s->a);
    measures[5] = 1.0 * sqrt(s->b);

    int ids[6], n = 0, total = 1;
    double meas[6];
    ids[n] = 0; meas[n++] = measures[0];
    total *= 10;
    if (p->type == RECTANGULAR || p->type == FLAT)
    {
        total *= 10;
        ids[n] = 1; meas[n++] = measures[1];
    }
    if (zAxis)
    {
        if (s->type == RECTANGULAR || s->type == FLAT)
        {
            total *= 10;
            ids[n] = 4; meas[n++] = measures[4];
        }
    }
    else
    {
        ids[n] = 3; meas[n++] = measures[3];
        total *= 10;
        if (s->type == RECTANGULAR)
        {
            total *= 100;
            ids[n] = 4; meas[n++] = measures[4];
            ids[n] = 5; meas[n++] = measures[5];
        }
        else if (s->type == THIN)
        {
            total *= 10;
            ids[n] = 5; meas[n++] = measures[5];
        }
        else if (s->type == FLAT)
        {
            total *= 10;
            ids[n] = 4; meas[n++] = measures[4];
        }
    }
    total = (int)((double)total * pow(2, pf - 1.0));
    /* the GPU cap applies to primary layers always and to secondary ones when pureGPU */
    int cappable[6] = {1, 1, 1, pureGPU, pureGPU, pureGPU};
    balance_with_cap(&total, &n, ids, meas, layer, gpu_cap, cappable);

    for (int i = 1; i < 6; ++i)
    {
        if (layer[i] == 1)
            layer[i] = (int)round((double)layer[0] * measures[i] / measures[0]);
        if (layer[i] == 0)
            layer[i] = 1;
        if (gpu_cap > 0 && layer[i] >= gpu_cap)
            layer[i] = gpu_cap;
    }
    int b[6], inc[6];
    for (int i = 0; i < 6; ++i)
        split_blocks(layer[i], &b[i], &inc[i]);
    *prim = make_args(b[0], b[1], b[2], inc[0], inc[1], inc[2]);
    *sec = make_args(b[3], b[4], b[5], inc[3], inc[4], inc[5]);
}

int oracle_pair_args(const double *pc, const double *sc, double pf, int gpu_cap, int zAxis, int pureGPU, int *out12)
{
    OCoil p, s;
    OArgs a, b;
    make_coil(pc, &p);
    make_coil(sc, &s);
    pair_args(&p, &s, sanitize_pf(pf), gpu_cap, zAxis, pureGPU, &a, &b);
    int v[12] = {a.aB, a.tB, a.lB, a.aI, a.tI, a.lI, b.aB, b.tB, b.lB, b.aI, b.tI, b.lI};
    memcpy(out12, v, sizeof v);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Field integrands (cylindrical, coil frame)                           */
/* ------------------------------------------------------------------ */
/* cos of the angular nodes over [0, pi], block by block
 * (CalculateFieldsFast.cxx:30-43) */
static double *angular_cos(const OArgs *u)
{
    double *cs = (double *)malloc(sizeof(double) * u->aB * u->aI);
    double blk = PI / u->aB;
    for (int j = 0; j < u->aB; ++j)
        for (int i = 0; i < u->aI; ++i)
            cs[j * u->aI + i] = cos(blk * (j + 0.5) + blk * 0.5 * g_pos[u->aI - 1][i]);
    return cs;
}

/* Coil::calculateAPotentialFast (src/Coil/Fields/CalculateFieldsFast.cxx:13-83) */
static double a_fast(const OCoil *k, double z, double r, const OArgs *u)
{
    double sum = 0.0;
    double tb = k->a / u->tB, ab = PI / u->aB;
    double cst = MI_REDUCED * k->J * tb * ab * 2 * 0.25;
    double top = z + k->b * 0.5, bot = z - k->b * 0.5;
    double *cs = angular_cos(u);
    for (int bt = 0; bt < u->tB; ++bt)
    {
        double bpos = k->R + tb * (bt + 0.5);
        for (int it = 0; it < u->tI; ++it)
        {
            double rt = bpos + tb * 0.5 * g_pos[u->tI - 1][it];
            double wt = g_wts[u->tI - 1][it];
            double cA = 2.0 * rt * r, cB = rt * rt + r * r;
            for (int bp = 0; bp < u->aB; ++bp)
                for (int ip = 0; ip < u->aI; ++ip)
                {
                    double wp = g_wts[u->aI - 1][ip];
                    double c = cs[bp * u->aI + ip];
                    double g = 1.0 / sqrt(cB - cA * c);
                    double d1 = top * g, d2 = bot * g;
                    double e1 = sqrt(d1 * d1 + 1.0), e2 = sqrt(d2 * d2 + 1.0);
                    double lg = log((e1 + d1) / (e2 + d2));
                    sum += cst * wt * wp * rt * c * lg;
                }
        }
    }
    free(cs);
    return sum;
}

/* Coil::calculateBFieldFast (CalculateFieldsFast.cxx:85-160) */
static void b_fast(const OCoil *k, double z, double r, const OArgs *u, double *H, double *Z)
{
    double h = 0.0, zz = 0.0;
    double tb = k->a / u->tB, ab = PI / u->aB;
    double cst = MI_REDUCED * k->J * tb * ab * 2 * 0.25;
    double top = z + k->b * 0.5, bot = z - k->b * 0.5;
    double *cs = angular_cos(u);
    for (int bt = 0; bt < u->tB; ++bt)
    {
        double bpos = k->R + tb * (bt + 0.5);
        for (int it = 0; it < u->tI; ++it)
        {
            double rt = bpos + tb * 0.5 * g_pos[u->tI - 1][it];
            double wt = g_wts[u->tI - 1][it];
            double cA = rt * rt, cB = rt * r, cC = cA + r * r;
            double d1 = top * top + cC, d2 = bot * bot + cC;
            double e = cst * wt;
            for (int bp = 0; bp < u->aB; ++bp)
                for (int ip = 0; ip < u->aI; ++ip)
                {
                    double wp = g_wts[u->aI - 1][ip];
                    double c = cs[bp * u->aI + ip];
                    double F = 2.0 * cB * c;
                    double g1 = 1.0 / sqrt(d1 - F), g2 = 1.0 / sqrt(d2 - F);
                    double hh = e * wp;
                    h += hh * rt * c * (g2 - g1);
                    zz += hh * ((cA - 0.5 * F) / (cC - F)) * (top * g1 - bot * g2);
                }
        }
    }
    free(cs);
    *H = h;
    *Z = zz;
}

/* Coil::calculateBGradientFast (CalculateFieldsFast.cxx:162-266);
 * out = {RPhi, RR, RZ, ZZ} */
static void g_fast(const OCoil *k, double z, double r, const OArgs *u, double *out)
{
    double rphi = 0, rr = 0, zzv = 0, rz = 0;
    double tb = k->a / u->tB, ab = PI / u->aB;
    double cst = MI_REDUCED * k->J * tb * ab * 2 * 0.25;
    double top = z + k->b * 0.5, bot = z - k->b * 0.5;
    double *cs = angular_cos(u);
    for (int bt = 0; bt < u->tB; ++bt)
    {
        double bpos = k->R + tb * (bt + 0.5);
        for (int it = 0; it < u->tI; ++it)
        {
            double rt = bpos + tb * 0.5 * g_pos[u->tI - 1][it];
            double wt = g_wts[u->tI - 1][it];
            double A = rt * rt, B = r * r, C = rt * r;
            double D = A + B, E = A * A + B * B, F = C * C;
            double G1 = D + top * top, G2 = D + bot * bot;
            double I = cst * wt;
            for (int bp = 0; bp < u->aB; ++bp)
                for (int ip = 0; ip < u->aI; ++ip)
                {
                    double wp = g_wts[u->aI - 1][ip];
                    double c = cs[bp * u->aI + ip];
                    double c2 = c * c;
                    double pe = 2 * C * c;
                    double J1 = G1 - pe, J2 = G2 - pe;
                    double K1 = sqrt(J1), K2 = sqrt(J2);
                    double L1 = 1 / (J1 * K1), L2 = 1 / (J2 * K2);
                    double M = D - pe;
                    double Nn = 2 * F * c * (c2 + 2.0) - C * (3 * c2 + 1) * D + c * E;
                    double O = c * D - 2 * C;
                    double Zf = I * wp;
                    rphi += Zf * (rt * c / r) * (1 / K2 - 1 / K1);
                    rr += Zf * (C - A * c) * c * (L1 - L2);
                    zzv += Zf * (A - C * c) * (L1 - L2);
                    rz += Zf * rt / (M * M) * (top * L1 * (O * J1 + Nn) - bot * L2 * (O * J2 + Nn));
                }
        }
    }
    free(cs);
    out[0] = rphi; out[1] = rr; out[2] = rz; out[3] = zzv;
}

/* Coil::calculateAPotentialSlow (src/Coil/Fields/CalculateFieldsSlow.cxx:13-84) */
static double a_slow(const OCoil *k, double z, double r, const OArgs *u)
{
    double sum = 0.0;
    double lb = k->b / u->lB, tb = k->a / u->tB, ab = PI / u->aB;
    double cst = MI_REDUCED * k->J * lb * tb * ab * 2 * 0.125;
    double *cs = angular_cos(u);
    for (int bl = 0; bl < u->lB; ++bl)
        for (int bt = 0; bt < u->tB; ++bt)
        {
            double lpos = -k->b * 0.5 + lb * (bl + 0.5);
            double tpos = k->R + tb * (bt + 0.5);
            for (int il = 0; il < u->lI; ++il)
                for (int it = 0; it < u->tI; ++it)
                {
                    double zl = lpos + lb * 0.5 * g_pos[u->lI - 1][il];
                    double rt = tpos + tb * 0.5 * g_pos[u->tI - 1][it];
                    double ws = g_wts[u->lI - 1][il] * g_wts[u->tI - 1][it];
                    double cA = 2.0 * rt * r;
                    double cB = rt * rt + r * r + (zl + z) * (zl + z);
                    for (int bp = 0; bp < u->aB; ++bp)
                        for (int ip = 0; ip < u->aI; ++ip)
                        {
                            double wp = g_wts[u->aI - 1][ip];
                            double c = cs[bp * u->aI + ip];
                            sum += cst * ws * wp * (rt * c) / sqrt(cB - cA * c);
                        }
                }
        }
    free(cs);
    return sum;
}

/* Coil::calculateBFieldSlow (CalculateFieldsSlow.cxx:86-165) */
static void b_slow(const OCoil *k, double z, double r, const OArgs *u, double *H, double *Z)
{
    double h = 0.0, zz = 0.0;
    double lb = k->b / u->lB, tb = k->a / u->tB, ab = PI / u->aB;
    double cst = MI_REDUCED * k->J * lb * tb * ab * 2 * 0.125;
    double *cs = angular_cos(u);
    for (int bl = 0; bl < u->lB; ++bl)
        for (int bt = 0; bt < u->tB; ++bt)
        {
            double lpos = -k->b * 0.5 + lb * (bl + 0.5);
            double tpos = k->R + tb * (bt + 0.5);
            for (int il = 0; il < u->lI; ++il)
                for (int it = 0; it < u->tI; ++it)
                {
                    double zl = lpos + lb * 0.5 * g_pos[u->lI - 1][il];
                    double rt = tpos + tb * 0.5 * g_pos[u->tI - 1][it];
                    double ws = g_wts[u->lI - 1][il] * g_wts[u->tI - 1][it];
                    double A = rt * rt, B = rt * (zl + z), C = rt * r;
                    double D = A + r * r + (zl + z) * (zl + z);
                    double E = cst * ws;
                    for (int bp = 0; bp < u->aB; ++bp)
                        for (int ip = 0; ip < u->aI; ++ip)
                        {
                            double wp = g_wts[u->aI - 1][ip];
                            double c = cs[bp * u->aI + ip];
                            double F = 2.0 * C * c;
                            double Hh = (D - F) * sqrt(D - F);
                            double G = E * wp / Hh;
                            zz += G * (A - C * c);
                            h += G * (B * c);
                        }
                }
        }
    free(cs);
    *H = h;
    *Z = zz;
}

/* Coil::calculateBGradientSlow (CalculateFieldsSlow.cxx:167-265) */
static void g_slow(const OCoil *k, double z, double r, const OArgs *u, double *out)
{
    double rphi = 0, rr = 0, zzv = 0, rz = 0;
    double lb = k->b / u->lB, tb = k->a / u->tB, ab = PI / u->aB;
    double cst = MI_REDUCED * k->J * lb * tb * ab * 2 * 0.125;
    double *cs = angular_cos(u);
    for (int bl = 0; bl < u->lB; ++bl)
        for (int bt = 0; bt < u->tB; ++bt)
        {
            double lpos = -k->b * 0.5 + lb * (bl + 0.5);
            double tpos = k->R + tb * (bt + 0.5);
            for (int il = 0; il < u->lI; ++il)
                for (int it = 0; it < u->tI; ++it)
                {
                    double zl = lpos + lb * 0.5 * g_pos[u->lI - 1][il];
                    double rt = tpos + tb * 0.5 * g_pos[u->tI - 1][it];
                    double ws = g_wts[u->lI - 1][il] * g_wts[u->tI - 1][it];
                    double A = rt * rt, B = r * r, C = (zl + z) * (zl + z);
                    double D = r * rt, E = rt * (zl + z), F = 1.0 / r;
                    double G = 2.0 * A + 2.0 * B - C, Hh = A + B + C;
                    double I = cst * ws;
                    for (int bp = 0; bp < u->aB; ++bp)
                        for (int ip = 0; ip < u->aI; ++ip)
                        {
                            double wp = g_wts[u->aI - 1][ip];
                            double c = cs[bp * u->aI + ip];
                            double J = Hh - 2.0 * D * c;
                            double K = J * J * sqrt(J);
                            double X = I * wp / (J * sqrt(J));
                            double Y = I * wp / K;
                            rphi += X * (F * E * c);
                            rr += Y * (-3.0 * E * (r - rt * c)) * c;
                            zzv += Y * (-3.0 * E * (rt - r * c));
                            rz += Y * (rt * (G - D * c) * c - 3.0 * A * r);
                        }
                }
        }
    free(cs);
    out[0] = rphi; out[1] = rr; out[2] = rz; out[3] = zzv;
}

/* ------------------------------------------------------------------ */
/* Cartesian wrappers (src/Coil/Fields/CalculateFieldsMethods.cxx)      */
/* ------------------------------------------------------------------ */
static void to_coil_frame(const OCoil *k, const double *p, double *z, double *r, double *phi)
{
    double d[3] = {p[0] - k->pos[0], p[1] - k->pos[1], p[2] - k->pos[2]};
    double x = k->Tinv[0] * d[0] + k->Tinv[1] * d[1] + k->Tinv[2] * d[2];
    double y = k->Tinv[3] * d[0] + k->Tinv[4] * d[1] + k->Tinv[5] * d[2];
    double zz = k->Tinv[6] * d[0] + k->Tinv[7] * d[1] + k->Tinv[8] * d[2];
    *z = zz;
    *r = sqrt(x * x + y * y);
    *phi = atan2(y, x);
}

static void matvec(const double *T, const double *v, double *o)
{
    o[0] = T[0] * v[0] + T[1] * v[1] + T[2] * v[2];
    o[1] = T[3] * v[0] + T[4] * v[1] + T[5] * v[2];
    o[2] = T[6] * v[0] + T[7] * v[1] + T[8] * v[2];
}

/* qty: 0 = A, 1 = B, 2 = E, 3 = G; out receives 3 or 9 doubles */
static void point_field(const OCoil *k, const OArgs *u, int qty, const double *p, double *out)
{
    double z, r, phi;
    to_coil_frame(k, p, &z, &r, &phi);
    if (qty == 0 || qty == 2)
    {
        double a = k->fast ? a_fast(k, z, r, u) : a_slow(k, z, r, u);
        double v[3] = {a * (-1) * sin(phi), a * cos(phi), 0.0};
        matvec(k->T, v, out);
        if (qty == 2)
            for (int i = 0; i < 3; ++i)
                out[i] *= 2 * PI * k->f;
    }
    else if (qty == 1)
    {
        double H, Z;
        if (k->fast) b_fast(k, z, r, u, &H, &Z);
        else b_slow(k, z, r, u, &H, &Z);
        double v[3] = {H * cos(phi), H * sin(phi), Z};
        matvec(k->T, v, out);
    }
    else
    {
        double b[4];
        if (k->fast) g_fast(k, z, r, u, b);
        else g_slow(k, z, r, u, b);
        double rphi = b[0], rr = b[1], rz = b[2], zz = b[3];
        double G[9];
        if (r / k->R < ZAXIS_RATIO)
        {
            double g[9] = {rr, 0, 0, 0, rr, 0, 0, 0, zz};
            memcpy(G, g, sizeof g);
        }
        else
        {
            double cp = cos(phi), sp = sin(phi);
            double xx = rr * cp * cp + rphi * sp * sp;
            double yy = rr * sp * sp + rphi * cp * cp;
            double xy = 0.5 * sin(2 * phi) * (rr - rphi);
            double xz = rz * cos(phi), yz = rz * sin(phi);
            double g[9] = {xx, xy, xz, xy, yy, yz, xz, yz, zz};
            memcpy(G, g, sizeof g);
        }
        /* the reference returns T * G, not T * G * T^-1 (CalculateFieldsMethods.cxx:83) */
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                out[3 * i + j] = k->T[3 * i] * G[j] + k->T[3 * i + 1] * G[3 + j] + k->T[3 * i + 2] * G[6 + j];
    }
}

/* One coil at n points with explicit precision args (prec6) or, when prec6 is
 * NULL, the coil's default CPU precision at pf. */
int oracle_coil_fields(const double *c, double pf, const int *prec6, int qty, long long n, const double *pts,
                       double *out)
{
    build_tables();
    OCoil k;
    make_coil(c, &k);
    OArgs u = prec6 ? make_args(prec6[0], prec6[1], prec6[2], prec6[3], prec6[4], prec6[5])
                    : coil_args(&k, sanitize_pf(pf), 0);
    int w = qty == 3 ? 9 : 3;
    for (long long i = 0; i < n; ++i)
        point_field(&k, &u, qty, pts + 3 * i, out + w * i);
    return 0;
}

/* CoilGroup::computeAll* with CPU_ST (src/CoilGroup/Fields/ComputeFields.cxx:60-71):
 * each member at its default CPU precision for pf, summed in member order */
int oracle_group_fields(int ncoils, const double *coils, double pf, int qty, long long n, const double *pts,
                        double *out)
{
    build_tables();
    int w = qty == 3 ? 9 : 3;
    memset(out, 0, sizeof(double) * (size_t)n * w);
    double tmp[9];
    for (int c = 0; c < ncoils; ++c)
    {
        OCoil k;
        make_coil(coils + 11 * c, &k);
        OArgs u = coil_args(&k, sanitize_pf(pf), 0);
        for (long long i = 0; i < n; ++i)
        {
            point_field(&k, &u, qty, pts + 3 * i, tmp);
            for (int j = 0; j < w; ++j)
                out[w * i + j] += tmp[j];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Coil pairs                                                           */
/* ------------------------------------------------------------------ */
/* Coil::isZAxisCase (src/Coil/Utils/SupportFunctions.cxx:55-70) */
static int z_axis_case(const OCoil *p, const OCoil *s)
{
    return fabs(p->pos[0] / p->R) < ZAXIS_RATIO && fabs(p->pos[1] / p->R) < ZAXIS_RATIO &&
           fabs(s->pos[0] / p->R) < ZAXIS_RATIO && fabs(s->pos[1] / p->R) < ZAXIS_RATIO &&
           fabs(p->yAngle / (2 * PI)) < ZAXIS_RATIO && fabs(s->yAngle / (2 * PI)) < ZAXIS_RATIO;
}

int oracle_z_axis_case(const double *pc, const double *sc)
{
    OCoil p, s;
    make_coil(pc, &p);
    make_coil(sc, &s);
    return z_axis_case(&p, &s);
}

static void cross(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

/* Coil::improvedPrecisionCase (SupportFunctions.cxx:124-161) */
static int improved_case(const OCoil *p, const OCoil *s, double *offset)
{
    double pn[3] = {sin(p->yAngle) * cos(p->zAngle), sin(p->yAngle) * sin(p->zAngle), cos(p->yAngle)};
    double sn[3] = {sin(s->yAngle) * cos(s->zAngle), sin(s->yAngle) * sin(s->zAngle), cos(s->yAngle)};
    double d[3] = {p->pos[0] - s->pos[0], p->pos[1] - s->pos[1], p->pos[2] - s->pos[2]};
    double pl[3];
    cross(pn, d, pl);
    double dot = pl[0] * sn[0] + pl[1] * sn[1] + pl[2] * sn[2];
    int improved = fabs(dot) <= PLANE_RATIO;
    *offset = 0.0;
    if (improved)
    {
        if (pl[0] == 0.0 && pl[1] == 0.0 && pl[2] == 0.0)
            cross(sn, d, pl);
        if (pl[0] == 0.0 && pl[1] == 0.0 && pl[2] == 0.0)
            cross(sn, pn, pl);
        *offset = atan2(cos(s->yAngle) * (pl[0] * cos(s->zAngle) + pl[1] * sin(s->zAngle)) - pl[2] * sin(s->yAngle),
                        pl[0] * sin(s->zAngle) - pl[1] * cos(s->zAngle));
    }
    return improved;
}

/* secondary node cloud shared by M and F/T
 * (CalculateMInductanceGeneral.cxx:35-103, CalculateForceGeneral.cxx:36-105,
 *  ring geometry from Coil::calculateRingIncrementPosition, SupportFunctions.cxx:72-122) */
typedef struct
{
    long long n;
    double *pos;   /* 3 per node */
    double *tan;   /* 3 per node */
    double *w;
} Cloud;

static Cloud sec_cloud(const OCoil *s, const OArgs *u, int improved, double offset)
{
    Cloud cl;
    int nring = u->aB * u->aI;
    double *ringP = (double *)malloc(sizeof(double) * 3 * nring);
    double *ringT = (double *)malloc(sizeof(double) * 3 * nring);
    double ablk = improved ? PI / u->aB : 2 * PI / u->aB;
    double sA = sin(s->yAngle), cA = cos(s->yAngle), sB = sin(s->zAngle), cB = cos(s->zAngle);
    for (int b = 0; b < u->aB; ++b)
        for (int i = 0; i < u->aI; ++i)
        {
            double ph = offset + ablk * (b + 0.5) + ablk * 0.5 * g_pos[u->aI - 1][i];
            double sp = sin(ph), cp = cos(ph);
            int q = b * u->aI + i;
            ringP[3 * q] = cB * cA * cp - sB * sp;
            ringP[3 * q + 1] = sB * cA * cp + cB * sp;
            ringP[3 * q + 2] = -sA * cp;
            ringT[3 * q] = -cB * cA * sp - sB * cp;
            ringT[3 * q + 1] = -sB * cA * sp + cB * cp;
            ringT[3 * q + 2] = sA * sp;
        }
    cl.n = (long long)u->lB * u->lI * u->tB * u->tI * nring;
    cl.pos = (double *)malloc(sizeof(double) * 3 * cl.n);
    cl.tan = (double *)malloc(sizeof(double) * 3 * cl.n);
    cl.w = (double *)malloc(sizeof(double) * cl.n);
    double lbs = s->b / u->lB, tbs = s->a / u->tB;
    long long q = 0;
    for (int zb = 0; zb < u->lB; ++zb)
        for (int rb = 0; rb < u->tB; ++rb)
        {
            double zbp = -s->b * 0.5 + lbs * (zb + 0.5);
            double rbp = s->R + tbs * (rb + 0.5);
            for (int zi = 0; zi < u->lI; ++zi)
                for (int ri = 0; ri < u->tI; ++ri)
                {
                    double rr = rbp + tbs * 0.5 * g_pos[u->tI - 1][ri];
                    double ld = zbp + lbs * 0.5 * g_pos[u->lI - 1][zi];
                    for (int pb = 0; pb < u->aB; ++pb)
                        for (int pi = 0; pi < u->aI; ++pi)
                        {
                            int ph = pb * u->aI + pi;
                            cl.pos[3 * q] = s->pos[0] + ld * sin(s->yAngle) * cos(s->zAngle) + rr * ringP[3 * ph];
                            cl.pos[3 * q + 1] = s->pos[1] + ld * sin(s->yAngle) * sin(s->zAngle) + rr * ringP[3 * ph + 1];
                            cl.pos[3 * q + 2] = s->pos[2] + ld * cos(s->yAngle) + rr * ringP[3 * ph + 2];
                            memcpy(cl.tan + 3 * q, ringT + 3 * ph, 3 * sizeof(double));
                            cl.w[q] = 0.125 * rr * g_wts[u->lI - 1][zi] * g_wts[u->tI - 1][ri] * g_wts[u->aI - 1][pi];
                            ++q;
                        }
                }
        }
    free(ringP);
    free(ringT);
    return cl;
}

static void free_cloud(Cloud *c)
{
    free(c->pos);
    free(c->tan);
    free(c->w);
}

/* Coil::calculateMutualInductanceGeneral (src/Coil/MInductance/CalculateMInductanceGeneral.cxx:8-117) */
static double m_general(const OCoil *p, const OCoil *s, const OArgs *pu, const OArgs *su)
{
    double offset;
    int improved = improved_case(p, s, &offset);
    Cloud cl = sec_cloud(s, su, improved, offset);
    double m = 0.0, a[3];
    for (long long i = 0; i < cl.n; ++i)
    {
        point_field(p, pu, 0, cl.pos + 3 * i, a);
        m += (a[0] * cl.tan[3 * i] + a[1] * cl.tan[3 * i + 1] + a[2] * cl.tan[3 * i + 2]) * cl.w[i];
    }
    free_cloud(&cl);
    m /= (su->lB * su->tB * su->aB);
    return m * 2 * PI * s->N / p->I;
}

/* Coil::calculateForceTorqueGeneral (src/Coil/ForceAndTorque/CalculateForceGeneral.cxx:9-131) */
static void ft_general(const OCoil *p, const OCoil *s, const OArgs *pu, const OArgs *su, double *out6)
{
    Cloud cl = sec_cloud(s, su, 0, 0.0);
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0}, b[3], dF[3], dT[3], rr[3];
    for (long long i = 0; i < cl.n; ++i)
    {
        point_field(p, pu, 1, cl.pos + 3 * i, b);
        cross(cl.tan + 3 * i, b, dF);
        for (int j = 0; j < 3; ++j)
        {
            dF[j] *= cl.w[i];
            F[j] += dF[j];
            rr[j] = cl.pos[3 * i + j] - s->pos[j];
        }
        cross(rr, dF, dT);
        for (int j = 0; j < 3; ++j)
            T[j] += dT[j];
    }
    free_cloud(&cl);
    double fac = 2 * PI * (s->I * s->N) / (su->lB * su->tB * su->aB);
    for (int j = 0; j < 3; ++j)
    {
        out6[j] = F[j] * fac;
        out6[3 + j] = T[j] * fac;
    }
}

/* ------------------------------------------------------------------ */
/* Coaxial pairs: the z-axis formulas                                   */
/* ------------------------------------------------------------------ */
/* Coil::calculateMutualInductanceZAxisFast (src/Coil/MInductance/CalculateMInductanceZAxis.cxx:87-232)
 * and Coil::calculateAmpereForceZAxisFast (src/Coil/ForceAndTorque/CalculateForceZAxis.cxx:85-219):
 * both length integrals in closed form; force != 0 selects the axial force. */
static double zaxis_fast(const OCoil *p, const OCoil *s, double zd, const OArgs *pu, const OArgs *su, int force)
{
    double tb = p->a / pu->tB, ab = PI / pu->aB, rb = s->a / su->tB;
    double constant = MI_REDUCED * p->J * s->J * tb * ab * rb * 0.125;
    double *cs = angular_cos(pu);
    zd -= p->pos[2];
    double z1 = zd + s->b * 0.5 + p->b * 0.5, z2 = zd + s->b * 0.5 - p->b * 0.5;
    double z3 = zd - s->b * 0.5 - p->b * 0.5, z4 = zd - s->b * 0.5 + p->b * 0.5;
    double z1s = z1 * z1, z2s = z2 * z2, z3s = z3 * z3, z4s = z4 * z4;
    double sum = 0.0;
    for (int bR = 0; bR < su->tB; ++bR)
    {
        double blockR = s->R + rb * (bR + 0.5);
        for (int iR = 0; iR < su->tI; ++iR)
        {
            double r = blockR + (rb * 0.5) * g_pos[su->tI - 1][iR];
            double wR = g_wts[su->tI - 1][iR];
            for (int bT = 0; bT < pu->tB; ++bT)
            {
                double blockT = p->R + tb * (bT + 0.5);
                for (int iT = 0; iT < pu->tI; ++iT)
                {
                    double t = blockT + (tb * 0.5) * g_pos[pu->tI - 1][iT];
                    double wT = g_wts[pu->tI - 1][iT];
                    double c0 = constant * wR * wT;
                    double A = 2.0 * t * r, B = t * t + r * r;
                    for (int bP = 0; bP < pu->aB; ++bP)
                        for (int iP = 0; iP < pu->aI; ++iP)
                        {
                            double wP = g_wts[pu->aI - 1][iP];
                            double c = cs[bP * pu->aI + iP];
                            double C = B - A * c, D = sqrt(C);
                            if (!force)
                            {
                                double E1 = sqrt(C + z1s), E2 = sqrt(C + z2s), E3 = sqrt(C + z3s), E4 = sqrt(C + z4s);
                                double F1 = z1 / D, F2 = z2 / D, F3 = z3 / D, F4 = z4 / D;
                                double G1 = sqrt(F1 * F1 + 1.0), G2 = sqrt(F2 * F2 + 1.0);
                                double G3 = sqrt(F3 * F3 + 1.0), G4 = sqrt(F4 * F4 + 1.0);
                                double H1 = z1 * log(F1 + G1), H2 = z2 * log(F2 + G2);
                                double H3 = z3 * log(F3 + G3), H4 = z4 * log(F4 + G4);
                                sum += c0 * wP * A * c * (H1 - H2 + H3 - H4 - E1 + E2 - E3 + E4);
                            }
                            else
                            {
                                double E1 = z1 / D, E2 = z2 / D, E3 = z3 / D, E4 = z4 / D;
                                double G1 = E1 + sqrt(E1 * E1 + 1.0), G2 = E2 + sqrt(E2 * E2 + 1.0);
                                double G3 = E3 + sqrt(E3 * E3 + 1.0), G4 = E4 + sqrt(E4 * E4 + 1.0);
                                sum += c0 * wP * A * c * log(G2 * G4 / (G1 * G3));
                            }
                        }
                }
            }
        }
    }
    free(cs);
    return force ? (-1.0) * sum * 2 * PI : sum * 2 * PI / (p->I * s->I);
}

/* Coil::calculateMutualInductanceZAxisSlow (CalculateMInductanceZAxis.cxx:17-85) and
 * Coil::calculateAmpereForceZAxisSlow (CalculateForceZAxis.cxx:16-83): the primary's
 * |A| (or B_x) on the secondary's (r, z) grid in the plane y = 0. */
static double zaxis_slow(const OCoil *p, const OCoil *s, double zd, const OArgs *pu, const OArgs *su, int force)
{
    double lbs = s->b / su->lB, tbs = s->a / su->tB;
    double sum = 0.0;
    for (int bZ = 0; bZ < su->lB; ++bZ)
        for (int bR = 0; bR < su->tB; ++bR)
        {
            double zBlock = (-1) * (s->b * 0.5) + lbs * (bZ + 0.5);
            double rBlock = s->R + tbs * (bR + 0.5);
            for (int iZ = 0; iZ < su->lI; ++iZ)
                for (int iR = 0; iR < su->tI; ++iR)
                {
                    double z = zd + zBlock + (lbs * 0.5) * g_pos[su->lI - 1][iZ];
                    double r = rBlock + (tbs * 0.5) * g_pos[su->tI - 1][iR];
                    double w = r * 0.25 * g_wts[su->lI - 1][iZ] * g_wts[su->tI - 1][iR];
                    double pt[3] = {r, 0.0, z}, v[3];
                    point_field(p, pu, force ? 1 : 0, pt, v);
                    sum += (force ? v[0] : sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])) * w;
                }
        }
    sum /= (su->lB * su->tB);
    return force ? (-1.0) * sum * 2 * PI * s->N * s->I : sum * 2 * PI * s->N / p->I;
}

static double zaxis_value(const OCoil *p, const OCoil *s, const OArgs *pu, const OArgs *su, int force)
{
    int fast = (p->type == RECTANGULAR || p->type == THIN) && (s->type == RECTANGULAR || s->type == THIN);
    return fast ? zaxis_fast(p, s, s->pos[2], pu, su, force) : zaxis_slow(p, s, s->pos[2], pu, su, force);
}

/* Mutual inductance with explicit pair args (args12) or, when args12 is NULL,
 * the CPU pair args at pf (z-axis arguments for a coaxial pair), dispatched as
 * Coil::computeMutualInductance (src/Coil/MInductance/ComputeMInductanceMethods.cxx:7-40). */
int oracle_mutual_inductance(const double *pc, const double *sc, double pf, const int *args12, double *out)
{
    build_tables();
    OCoil p, s;
    make_coil(pc, &p);
    make_coil(sc, &s);
    int zax = z_axis_case(&p, &s);
    OArgs pu, su;
    if (args12)
    {
        pu = make_args(args12[0], args12[1], args12[2], args12[3], args12[4], args12[5]);
        su = make_args(args12[6], args12[7], args12[8], args12[9], args12[10], args12[11]);
    }
    else
        pair_args(&p, &s, sanitize_pf(pf), 0, zax, 0, &pu, &su);
    *out = zax ? zaxis_value(&p, &s, &pu, &su, 0) : m_general(&p, &s, &pu, &su);
    return 0;
}

int oracle_force_torque(const double *pc, const double *sc, double pf, const int *args12, double *out6)
{
    build_tables();
    OCoil p, s;
    make_coil(pc, &p);
    make_coil(sc, &s);
    int zax = z_axis_case(&p, &s);
    OArgs pu, su;
    if (args12)
    {
        pu = make_args(args12[0], args12[1], args12[2], args12[3], args12[4], args12[5]);
        su = make_args(args12[6], args12[7], args12[8], args12[9], args12[10], args12[11]);
    }
    else
        pair_args(&p, &s, sanitize_pf(pf), 0, zax, 0, &pu, &su);
    if (zax)
    {
        /* Coil::computeForceTorque (src/Coil/ForceAndTorque/ComputeForceMethods.cxx:4-23) */
        for (int i = 0; i < 6; ++i)
            out6[i] = 0.0;
        out6[2] = zaxis_value(&p, &s, &pu, &su, 1);
    }
    else
        ft_general(&p, &s, &pu, &su, out6);
    return 0;
}

/* Self inductance, Coil::computeAndSetSelfInductance
 * (src/Coil/MInductance/ComputeMInductanceMethods.cxx:55-81): the centred coil,
 * its z-axis pair arguments with itself (or args12); FLAT through the coaxial
 * mutual inductance with itself, RECTANGULAR / THIN through the closed form of
 * Coil::calculateSelfInductance (src/Coil/MInductance/CalculateMInductanceZAxis.cxx:233-319).
 * Returns 1 for a FILAMENT (divergent integral). */
int oracle_self_inductance(const double *c, double pf, const int *args12, double *out)
{
    build_tables();
    double row[11];
    for (int i = 0; i < 11; ++i)
        row[i] = c[i];
    row[6] = row[7] = row[8] = row[9] = row[10] = 0.0;
    OCoil k;
    make_coil(row, &k);
    if (k.type == FILAMENT)
        return 1;
    OArgs pu, su;
    if (args12)
    {
        pu = make_args(args12[0], args12[1], args12[2], args12[3], args12[4], args12[5]);
        su = make_args(args12[6], args12[7], args12[8], args12[9], args12[10], args12[11]);
    }
    else
        pair_args(&k, &k, sanitize_pf(pf), 0, 1, 0, &pu, &su);
    if (k.type == FLAT)
    {
        *out = zaxis_value(&k, &k, &pu, &su, 0);
        return 0;
    }
    double tb = k.a / pu.tB, ab = PI / pu.aB, rb = 1.0 / su.tB;
    double constant = MI_REDUCED * k.J * tb * ab * rb * 2 * 0.125;
    double b2 = k.b * k.b;
    double *cs = angular_cos(&pu);
    double sum = 0.0;
    for (int bR = 0; bR < su.tB; ++bR)
    {
        double blockR = k.R + rb * k.a * (bR + 0.5);
        for (int iR = 0; iR < su.tI; ++iR)
        {
            double r = blockR + (rb * k.a * 0.5) * g_pos[su.tI - 1][iR];
            double wR = g_wts[su.tI - 1][iR];
            for (int bT = 0; bT < pu.tB; ++bT)
            {
                double blockT = k.R + tb * (bT + 0.5);
                for (int iT = 0; iT < pu.tI; ++iT)
                {
                    double t = blockT + (tb * 0.5) * g_pos[pu.tI - 1][iT];
                    double wT = g_wts[pu.tI - 1][iT];
                    double c0 = constant * wR * wT;
                    double A = 2 * t * r, B = t * t + r * r;
                    for (int bP = 0; bP < pu.aB; ++bP)
                        for (int iP = 0; iP < pu.aI; ++iP)
                        {
                            double wP = g_wts[pu.aI - 1][iP];
                            double cc = cs[bP * pu.aI + iP];
                            double C = B - A * cc;
                            double D = sqrt(C), E = sqrt(C + b2);
                            double F = k.b / D, G = sqrt(F * F + 1.0), H = log(F + G);
                            sum += c0 * wP * A * cc * (D - E + k.b * H);
                        }
                }
            }
        }
    }
    free(cs);
    *out = sum * 2 * PI * k.N / (k.I * k.b);
    return 0;
}
