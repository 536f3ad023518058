// Host-side coil set-up, Gauss-Legendre tables and precision balancing.
//
// The increment balancing must agree with the reference bit for bit (the node
// counts decide which quadrature is evaluated), so the floating-point steps
// follow the reference's order of operations:
//   PrecisionArguments::calculatePrecisionArguments
//       src/Coil/PrecisionArguments/PrecisionArguments.cxx:69-185
//   CoilPairArguments::balanceIncrements / getAppropriateCoilPairArguments
//       src/Coil/PrecisionArguments/CoilPairArguments.cxx:20-255
//   Coil::Coil, calculateCoilType, calculateTransformationMatrices
//       src/Coil/Coil.cxx:46-67, src/Coil/Utils/CalculateAttributes.cxx:50-78
#include "ccoil_internal.h"

#include <cmath>
#include <cstring>
#include <mutex>

namespace ccoil
{
namespace
{
constexpr double kThinRatio = 1e-7;        // g_thinCoilApproximationRatio
constexpr double kPrimModifier = 1.414213562; // g_primAngularWeightModifier = g_primLinearWeightModifier
constexpr double kSecModifier = 1.0;         // g_secAngularWeightModifier = g_secLinearWeightModifier
constexpr int kBaseIncrements = 10;          // g_baseLayerIncrementsCPU = g_baseLayerIncrementsGPU
constexpr int kDefaultOrder = 20;
constexpr double kPi = 3.14159265358979323846;

double g_nodes[kMaxOrder][kMaxOrder];
double g_weights[kMaxOrder][kMaxOrder];
std::once_flag g_tables_once;

void legendreValue(int n, long double x, long double &p, long double &dp)
{
    long double prev = 1.0L, cur = x;
    for (int k = 2; k <= n; ++k)
    {
        long double next = ((2.0L * k - 1.0L) * x * cur - (k - 1.0L) * prev) / k;
        prev = cur;
        cur = next;
    }
    if (n == 0)
    {
        p = 1.0L;
        dp = 0.0L;
        return;
    }
    p = cur;
    dp = n * (x * cur - prev) / (x * x - 1.0L);
}

// Newton iteration on P_n in extended precision from the asymptotic root
// estimate cos(pi (i + 3/4) / (n + 1/2)); nodes mirrored so the table is exactly
// symmetric, weights w = 2 / ((1 - x^2) P_n'(x)^2).
void buildTables()
{
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int n = 1; n <= kMaxOrder; ++n)
    {
        for (int i = 0; i < n / 2; ++i)
        {
            long double x = std::cos(pi * (i + 0.75L) / (n + 0.5L));
            long double p, dp;
            for (int it = 0; it < 100; ++it)
            {
                legendreValue(n, x, p, dp);
                long double step = p / dp;
                x -= step;
                if (std::fabs(step) < 1e-22L)
                    break;
            }
            legendreValue(n, x, p, dp);
            long double w = 2.0L / ((1.0L - x * x) * dp * dp);
            g_nodes[n - 1][n - 1 - i] = double(x);
            g_nodes[n - 1][i] = -double(x);
            g_weights[n - 1][n - 1 - i] = double(w);
            g_weights[n - 1][i] = double(w);
        }
        if (n % 2 == 1)
        {
            long double p, dp;
            legendreValue(n, 0.0L, p, dp);
            g_nodes[n - 1][n / 2] = 0.0;
            g_weights[n - 1][n / 2] = double(2.0L / (dp * dp));
        }
    }
}

PrecisionArgs clampArgs(int aB, int tB, int lB, int aI, int tI, int lI)
{
    // PrecisionArguments::PrecisionArguments(int ...) (PrecisionArguments.cxx:29-54),
    // including its use of the unclamped length increments for the length-block test
    PrecisionArgs r{aB, tB, lB, aI, tI, lI};
    if (aI > kMaxOrder || aI < 1) r.angular_increments = kDefaultOrder;
    if (tI > kMaxOrder || tI < 1) r.thickness_increments = kDefaultOrder;
    if (lI > kMaxOrder || lI < 1) r.length_increments = kDefaultOrder;
    if (aB < 1) r.angular_blocks = 1;
    if (tB < 1) r.thickness_blocks = 1;
    if (lI < 1) r.length_blocks = 1;
    return r;
}

// components: (layer id, measure) pairs in the reference's insertion order
struct Components
{
    int id[6];
    double measure[6];
    int count = 0;
    void add(int i, double m)
    {
        id[count] = i;
        measure[count] = m;
        ++count;
    }
    void erase(int k)
    {
        for (int j = k; j + 1 < count; ++j)
        {
            id[j] = id[j + 1];
            measure[j] = measure[j + 1];
        }
        --count;
    }
};

void balanceIncrements(int total, const Components &c, int *counts)
{
    if (c.count < 2)
    {
        counts[0] = total;
        return;
    }
    double effective = 1.0;
    for (int i = 0; i < c.count; ++i)
        effective *= c.measure[i];
    effective /= double(total);
    double linear = std::pow(effective, 1.0 / double(c.count));
    for (int i = 0; i < c.count; ++i)
        counts[i] = int(std::round(c.measure[i] / linear));
}

// The spill loop: a component above the GPU cap is pinned at the cap, removed,
// the total shrinks by the cap and the rest is rebalanced.  cappable[id] says
// which layers the cap applies to.
void balanceWithCap(int total, Components c, int cap, const bool *cappable, int *layer)
{
    int counts[6];
    bool spill;
    do
    {
        balanceIncrements(total, c, counts);
        spill = false;
        if (cap > 0)
        {
            for (int i = 0; i < c.count; ++i)
            {
                if (counts[i] > cap && cappable[c.id[i]])
                {
                    layer[c.id[i]] = cap;
                    for (int j = i; j + 1 < c.count; ++j)
                        counts[j] = counts[j + 1];
                    c.erase(i);
                    total = int(std::ceil(double(total) / double(cap)));
                    spill = true;
                    break;
                }
            }
        }
    } while (spill && c.count > 0);
    for (int i = 0; i < c.count; ++i)
        layer[c.id[i]] = counts[i];
}

void splitBlocks(int layer, int &blocks, int &incs)
{
    blocks = (layer - 1) / kMaxOrder + 1;
    incs = blocks > 1 ? layer / blocks + 1 : layer;
}

double sanitizeFactor(double pf) { return (pf < 1.0 || pf > 15.0) ? 5.0 : pf; }
} // namespace

const double *legendreNodes(int order)
{
    std::call_once(g_tables_once, buildTables);
    return g_nodes[order - 1];
}

const double *legendreWeights(int order)
{
    std::call_once(g_tables_once, buildTables);
    return g_weights[order - 1];
}

PrecisionArgs coilPrecision(const Coil &coil, double pf, int gpuCap)
{
    pf = sanitizeFactor(pf);
    int layer[3] = {1, 1, 1};
    double measures[3];
    measures[0] = kPrimModifier * std::sqrt(kPi * (coil.inner_radius + 0.5 * coil.thickness));
    measures[1] = kPrimModifier * std::sqrt(coil.thickness);
    measures[2] = kPrimModifier * std::sqrt(coil.length);

    Components c;
    int total = 1;
    c.add(0, measures[0]);
    total *= kBaseIncrements;
    if (coil.coil_type == kRectangular || coil.coil_type == kFlat)
    {
        total *= kBaseIncrements;
        c.add(1, measures[1]);
    }
    total = int(double(total) * std::pow(2, pf - 1.0));
    const bool cappable[6] = {true, true, true, true, true, true};
    balanceWithCap(total, c, gpuCap, cappable, layer);

    if (layer[2] == 1)
        layer[2] = int(std::round(double(layer[0]) * measures[2] / measures[0]));
    if (layer[2] == 0)
        layer[2] = 1;
    if (gpuCap > 0 && layer[2] > gpuCap)
        layer[2] = gpuCap;

    int b[3], n[3];
    for (int i = 0; i < 3; ++i)
        splitBlocks(layer[i], b[i], n[i]);
    return clampArgs(b[0], b[1], b[2], n[0], n[1], n[2]);
}

void pairPrecision(const Coil &prim, const Coil &sec, double pf, int gpuCap, bool zAxis, bool pureGPU,
                   PrecisionArgs &primOut, PrecisionArgs &secOut)
{
    pf = sanitizeFactor(pf);
    int layer[6] = {1, 1, 1, 1, 1, 1};
    double measures[6];
    measures[0] = kPrimModifier * std::sqrt(kPi * (prim.inner_radius + 0.5 * prim.thickness));
    measures[1] = kPrimModifier * std::sqrt(prim.thickness);
    measures[2] = kPrimModifier * std::sqrt(prim.length);
    measures[3] = kSecModifier * std::sqrt(2 * kPi * (sec.inner_radius + 0.5 * sec.thickness));
    measures[4] = kSecModifier * std::sqrt(sec.thickness);
    measures[5] = kSecModifier * std::sqrt(sec.length);

    Components c;
    int total = 1;
    c.add(0, measures[0]);
    total *= kBaseIncrements;
    if (prim.coil_type == kRectangular || prim.coil_type == kFlat)
    {
        total *= kBaseIncrements;
        c.add(1, measures[1]);
    }
    if (zAxis)
    {
        if (sec.coil_type == kRectangular || sec.coil_type == kFlat)
        {
            total *= kBaseIncrements;
            c.add(4, measures[4]);
        }
    }
    else
    {
        c.add(3, measures[3]);
        total *= kBaseIncrements;
        if (sec.coil_type == kRectangular)
        {
            total *= kBaseIncrements * kBaseIncrements;
            c.add(4, measures[4]);
            c.add(5, measures[5]);
        }
        else if (sec.coil_type == kThin)
        {
            total *= kBaseIncrements;
            c.add(5, measures[5]);
        }
        else if (sec.coil_type == kFlat)
        {
            total *= kBaseIncrements;
            c.add(4, measures[4]);
        }
    }
    total = int(double(total) * std::pow(2, pf - 1.0));
    const bool cappable[6] = {true, true, true, pureGPU, pureGPU, pureGPU};
    balanceWithCap(total, c, gpuCap, cappable, layer);

    for (int i = 1; i < 6; ++i)
    {
        if (layer[i] == 1)
            layer[i] = int(std::round(double(layer[0]) * measures[i] / measures[0]));
        if (layer[i] == 0)
            layer[i] = 1;
        if (gpuCap > 0 && layer[i] >= gpuCap)
            layer[i] = gpuCap;
    }
    int b[6], n[6];
    for (int i = 0; i < 6; ++i)
        splitBlocks(layer[i], b[i], n[i]);
    primOut = clampArgs(b[0], b[1], b[2], n[0], n[1], n[2]);
    secOut = clampArgs(b[3], b[4], b[5], n[3], n[4], n[5]);
}

void initCoil(double R, double a, double b, int N, double I, double f, const double pos[3], double yAngle,
              double zAngle, Coil &out)
{
    std::memset(&out, 0, sizeof(out));
    out.inner_radius = R;
    out.thickness = a / R < kThinRatio ? 1e-18 * R * kThinRatio : a;
    out.length = b / R < kThinRatio ? 1e-18 * R * kThinRatio : b;
    out.num_turns = N;
    out.use_fast_method = (b / R >= kThinRatio) ? 1 : 0;
    out.current = I;
    out.current_density = I * N / (out.length * out.thickness);
    out.sine_frequency = f > 0.0 ? f : 0.0;
    for (int i = 0; i < 3; ++i)
        out.position[i] = pos ? pos[i] : 0.0;
    out.y_axis_angle = yAngle;
    out.z_axis_angle = zAngle;

    bool thinA = out.thickness / R < kThinRatio, thinB = out.length / R < kThinRatio;
    out.coil_type = (thinA && thinB) ? kFilament : thinA ? kThin : thinB ? kFlat : kRectangular;

    double cY = std::cos(yAngle), sY = std::sin(yAngle), cZ = std::cos(zAngle), sZ = std::sin(zAngle);
    const double T[9] = {cZ * cZ * cY - sZ * sZ, -sZ * cZ * cY - sZ * cZ, cZ * sY,
                         sZ * cZ * cY + sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY,
                         -sY * cZ, sY * sZ, cY};
    const double Ti[9] = {cZ * cZ * cY - sZ * sZ, sZ * cZ * cY + sZ * cZ, -cZ * sY,
                          -sZ * cZ * cY - sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY,
                          sY * cZ, sY * sZ, cY};
    std::memcpy(out.transform, T, sizeof(T));
    std::memcpy(out.inverse_transform, Ti, sizeof(Ti));
}

bool validArgs(const PrecisionArgs &p)
{
    return p.angular_blocks >= 1 && p.thickness_blocks >= 1 && p.length_blocks >= 1 && p.angular_increments >= 1 &&
           p.angular_increments <= kMaxOrder && p.thickness_increments >= 1 &&
           p.thickness_increments <= kMaxOrder && p.length_increments >= 1 && p.length_increments <= kMaxOrder;
}
} // namespace ccoil
