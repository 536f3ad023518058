// Builds the per-coil node tables ("segments") that the field kernels stage
// into shared memory.  The node positions and weights are those of the
// reference's integrators:
//   fast method: src/Coil/Fields/CalculateFieldsFast.cxx:17-55  (thickness x angle)
//   slow method: src/Coil/Fields/CalculateFieldsSlow.cxx:17-66  (length x thickness x angle)
// with the per-layer block subdivision of the reference, the overall constant
// folded into the thickness weights, and the angular nodes on [0, pi]
// (cosine is even, so the reference integrates half the turn and doubles it).
#include "ccoil_internal.h"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace ccoil
{
namespace
{
constexpr double kPi = 3.14159265358979323846;
constexpr double kMuReduced = 1e-7;  // g_MiReduced
constexpr double kDefaultNearMargin = 0.1;

struct Entry
{
    double a, b;
};

// Margin of the FP32 path's near-field box, as a multiple of the coil's inner
// radius.  CCOIL_NEAR_MARGIN overrides it (a tuning knob read at plan creation).
double nearMargin()
{
    const char *env = std::getenv("CCOIL_NEAR_MARGIN");
    if (env)
    {
        double v = std::atof(env);
        if (v >= 0.0 && v < 100.0)
            return v;
    }
    return kDefaultNearMargin;
}

void appendBytes(std::vector<unsigned char> &blob, const void *p, size_t n)
{
    const unsigned char *c = static_cast<const unsigned char *>(p);
    blob.insert(blob.end(), c, c + n);
}
} // namespace

// Entry k of the FP32 angular pair table: node k of the FP64 table (in the
// reference's order) and its mirror n-1-k.  Both nodes' 1 - cos come from
// half-angle sines (no cancellation near phi = 0 or pi); the difference weight
// w2c2 is formed from their FP32 values, so it matches the squared distances
// the kernels build from them; an odd table's middle node is an entry of its
// own with half its weight.
PhiNode32 phiPair32(const PrecisionArgs &p, int k)
{
    const double aBlock = kPi / p.angular_blocks;
    const double *ax = legendreNodes(p.angular_increments), *aw = legendreWeights(p.angular_increments);
    const int n = p.angular_blocks * p.angular_increments;
    auto phiOf = [&](int j) {
        return aBlock * (j / p.angular_increments + 0.5) + (aBlock * 0.5) * ax[j % p.angular_increments];
    };
    const int m = n - 1 - k;
    const double w = aw[k % p.angular_increments];
    const double s = std::sin(0.5 * phiOf(k)), sm = std::sin(0.5 * phiOf(m));
    PhiNode32 e;
    e.omc = (float)(2.0 * s * s);
    if (m == k)
    {
        e.omcm = e.omc;
        e.w2c2 = 0.0f;
        e.wc = 0.0f;
        e.w = (float)(0.5 * w);
    }
    else
    {
        e.omcm = (float)(2.0 * sm * sm);
        const double twoC = (double)e.omcm - (double)e.omc;
        e.w2c2 = (float)(0.5 * w * twoC * twoC);
        e.wc = (float)(0.5 * w * twoC);
        e.w = (float)w;
    }
    e.ws2 = (float)((double)e.w * (double)e.omc * (double)e.omcm);
    return e;
}

void packPhiPairs2(const PhiNode32 *pairs, int count, std::vector<PhiPair2> &out)
{
    out.resize((size_t)(count + 1) / 2);
    for (int m = 0; 2 * m < count; ++m)
    {
        const PhiNode32 &a = pairs[2 * m];
        const PhiNode32 &b =
            2 * m + 1 < count ? pairs[2 * m + 1] : PhiNode32{0.0f, a.omc, a.omcm, 0.0f, 0.0f, 0.0f};
        out[m].omc = make_float2(a.omc, b.omc);
        out[m].omcm = make_float2(a.omcm, b.omcm);
        out[m].w = make_float2(a.w, b.w);
        out[m].w2c2 = make_float2(a.w2c2, b.w2c2);
        out[m].wc = make_float2(a.wc, b.wc);
        out[m].ws2 = make_float2(a.ws2, b.ws2);
    }
}

void buildPhiPairs32(const PrecisionArgs &p, std::vector<PhiNode32> &pairs)
{
    const int n = p.angular_blocks * p.angular_increments;
    pairs.resize((n + 1) / 2);
    for (int k = 0; k < (n + 1) / 2; ++k)
        pairs[k] = phiPair32(p, k);
}

// Near-field region of the FP32 path: the winding's cross-section box in
// (r, z), inflated by a margin; points inside are integrated in FP64.
void setNearBox(const Coil &k, SegmentHeader &h)
{
    const double margin = nearMargin() * k.inner_radius;
    h.near_lo[0] = k.inner_radius - margin;
    h.near_hi[0] = k.inner_radius + k.thickness + margin;
    h.near_lo[1] = -0.5 * k.length - margin;
    h.near_hi[1] = 0.5 * k.length + margin;
    h.near_r2 = margin * margin;
}

bool buildFieldSegments(const Coil *coils, int count, int field, int precision, SegmentSink &out, std::string &err)
{
    const bool fp32 = precision == CCOIL_PRECISION_FP32_COMPENSATED;

    for (int ci = 0; ci < count; ++ci)
    {
        const Coil &k = coils[ci];
        const PrecisionArgs &p = k.precision;
        if (!validArgs(p))
        {
            err = "coil " + std::to_string(ci) + ": precision arguments out of range (increments 1..100, blocks >= 1)";
            return false;
        }
        if (!(k.inner_radius > 0.0) || !(k.thickness > 0.0) || !(k.length > 0.0))
        {
            err = "coil " + std::to_string(ci) + ": inner radius, thickness and length must be positive";
            return false;
        }
        const bool fast = k.use_fast_method != 0;

        // thickness nodes with the overall constant folded in
        const double tBlock = k.thickness / p.thickness_blocks;
        const double aBlock = kPi / p.angular_blocks;
        double constant;
        if (fast)
            constant = kMuReduced * k.current_density * tBlock * aBlock * 2 * 0.25;
        else
            constant = kMuReduced * k.current_density * (k.length / p.length_blocks) * tBlock * aBlock * 2 * 0.125;

        std::vector<Entry> tNodes;
        const double *tx = legendreNodes(p.thickness_increments), *tw = legendreWeights(p.thickness_increments);
        for (int bt = 0; bt < p.thickness_blocks; ++bt)
        {
            double blockPos = k.inner_radius + tBlock * (bt + 0.5);
            for (int i = 0; i < p.thickness_increments; ++i)
                tNodes.push_back({blockPos + (tBlock * 0.5) * tx[i], constant * tw[i]});
        }
        std::vector<Entry> lNodes;
        if (!fast)
        {
            const double lBlock = k.length / p.length_blocks;
            const double *lx = legendreNodes(p.length_increments), *lw = legendreWeights(p.length_increments);
            for (int bl = 0; bl < p.length_blocks; ++bl)
            {
                double blockPos = -k.length * 0.5 + lBlock * (bl + 0.5);
                for (int i = 0; i < p.length_increments; ++i)
                    lNodes.push_back({blockPos + (lBlock * 0.5) * lx[i], lw[i]});
            }
        }
        // angular nodes over [0, pi]; cos(phi) = -sin(pi x / 2 ...) form is not
        // used here: the FP64 tables follow the reference's cos(block centre + ...)
        std::vector<Entry> phiNodes;
        std::vector<PhiNode32> phi32;
        const double *ax = legendreNodes(p.angular_increments), *aw = legendreWeights(p.angular_increments);
        for (int bp = 0; bp < p.angular_blocks; ++bp)
        {
            double blockPos = aBlock * (bp + 0.5);
            for (int i = 0; i < p.angular_increments; ++i)
                phiNodes.push_back({std::cos(blockPos + (aBlock * 0.5) * ax[i]), aw[i]});
        }
        if (fp32)
        {
            // FP32 mode: the FP64 table (used by the near-field pass) in mirror-pair
            // order, so that every segment's FP64 and FP32 tables cover the same nodes
            std::vector<Entry> paired(phiNodes.size());
            for (size_t j = 0; j < phiNodes.size(); ++j)
                paired[j] = phiNodes[pairOrderNode((int)j, (int)phiNodes.size())];
            phiNodes.swap(paired);
            buildPhiPairs32(p, phi32);
        }

        const int headerBytes = (int)sizeof(SegmentHeader);
        const int fixedBytes = headerBytes + 16 * (int)(tNodes.size() + lNodes.size());
        // FP32 mode: 16 bytes per FP64 node plus 48 per two mirror pairs, and
        // segments cut at multiples of four nodes so that no pair, and no packed
        // entry of two pairs, is split
        const int maxPhi = fp32 ? 4 * ((kSegmentBytes - fixedBytes) / (64 + (int)sizeof(PhiPair2)))
                                : (kSegmentBytes - fixedBytes) / 16;
        if (maxPhi < 1)
        {
            err = "coil " + std::to_string(ci) + ": thickness/length node tables exceed one staging segment";
            return false;
        }
        const int nPhi = (int)phiNodes.size();
        for (int start = 0; start < nPhi; start += maxPhi)
        {
            int cnt = std::min(maxPhi, nPhi - start);
            SegmentHeader h;
            std::memset(&h, 0, sizeof(h));
            for (int i = 0; i < 3; ++i)
                h.position[i] = k.position[i];
            std::memcpy(h.inv_transform, k.inverse_transform, sizeof(h.inv_transform));
            std::memcpy(h.transform, k.transform, sizeof(h.transform));
            h.half_length = k.length * 0.5;
            h.field_factor = field == CCOIL_FIELD_E ? 2 * kPi * k.sine_frequency : 1.0;
            h.inner_radius = k.inner_radius;
            h.n_t = (int)tNodes.size();
            h.n_l = (int)lNodes.size();
            h.n_phi = cnt;
            h.fast = fast ? 1 : 0;
            h.off_t = headerBytes / 16;
            h.off_l = h.off_t + h.n_t;
            h.off_phi = h.off_l + h.n_l;
            h.off_f32 = fp32 ? h.off_phi + cnt : 0;
            setNearBox(k, h);

            SegmentDesc d;
            d.offset = (long long)out.size();
            d.coil = ci;
            bool ok = out.append(&h, sizeof(h)) && out.append(tNodes.data(), 16 * tNodes.size()) &&
                      out.append(lNodes.data(), 16 * lNodes.size()) &&
                      out.append(phiNodes.data() + start, 16 * (size_t)cnt);
            if (ok && fp32)
            {
                std::vector<PhiPair2> packed;
                packPhiPairs2(phi32.data() + start / 2, (cnt + 1) / 2, packed);
                ok = out.append(packed.data(), sizeof(PhiPair2) * packed.size());
            }
            d.bytes = (int)((long long)out.size() - d.offset);
            if (!ok || !out.segment(d))
            {
                err = out.overflowMessage();
                return false;
            }
        }
    }
    return true;
}

namespace
{
// The plan path's sink: growable host vectors.
struct VectorSink final : SegmentSink
{
    SegmentSet &set;
    explicit VectorSink(SegmentSet &s) : set(s) {}
    bool append(const void *p, size_t n) override
    {
        appendBytes(set.blob, p, n);
        return true;
    }
    size_t size() const override { return set.blob.size(); }
    bool segment(const SegmentDesc &d) override
    {
        set.max_bytes = std::max(set.max_bytes, d.bytes);
        set.segs.push_back(d);
        return true;
    }
    std::string overflowMessage() const override { return "segment tables could not be stored"; }
};
} // namespace

bool buildFieldSegments(const Coil *coils, int count, int field, int precision, SegmentSet &out, std::string &err)
{
    out.blob.clear();
    out.segs.clear();
    out.max_bytes = 0;
    VectorSink sink(out);
    return buildFieldSegments(coils, count, field, precision, sink, err);
}
} // namespace ccoil
