// Coaxial coil pairs (included by pairs.cu inside its anonymous namespace).
//
// For a pair that Coil::isZAxisCase accepts (src/Coil/Utils/SupportFunctions.cxx:55-70:
// both centres on the primary's axis and both y axis angles zero, to 1e-12),
// the reference's CPU path does not use the general quadrature: it dispatches
// to z-axis formulas with pair arguments computed for the z-axis case
// (Coil::computeMutualInductance, src/Coil/MInductance/ComputeMInductanceMethods.cxx:7-30;
// Coil::computeForceTorque, src/Coil/ForceAndTorque/ComputeForceMethods.cxx:4-23):
//
//   both coils THIN or RECTANGULAR ("fast"): the two length integrals in closed
//     form, a triple sum over the secondary's radial nodes, the primary's
//     thickness nodes and the primary's angular nodes
//     (calculateMutualInductanceZAxisFast, CalculateMInductanceZAxis.cxx:87-232;
//      calculateAmpereForceZAxisFast, CalculateForceZAxis.cxx:85-219);
//   otherwise ("slow"): the primary's A (or B) at the secondary's (r, z) grid in
//     the plane y = 0, |A| (or B_x) summed with weights 0.25 r w_l w_r
//     (calculateMutualInductanceZAxisSlow, CalculateMInductanceZAxis.cxx:17-85;
//      calculateAmpereForceZAxisSlow, CalculateForceZAxis.cxx:16-83).
//
// Each term is evaluated with the reference's sequence of IEEE operations
// (the fast formulas cancel between their four length-limit terms).  The force
// is axial: (0, 0, Fz), torque zero.  A z-axis pair is skipped by the general
// kernel and recorded; zAxisKernel then adds the z-axis value of every
// coaxial primary, in primary order, to the arrangement's output.

struct alignas(16) ZAxisHeader
{
    SegmentHeader prim;    // primary field tables at the z-axis precision (slow formulas)
    double fast_constant;  // g_MiReduced J1 J2 tBlock aBlock rBlock 0.125
    double prim_length, sec_length;
    double prim_current, sec_current;
    double sec_turns;
    int fast;              // both coils THIN / RECTANGULAR
    int n_r, n_t, n_phi;   // fast: secondary radial, primary thickness, primary angular nodes
    int n_sl, n_st;        // slow: secondary length and thickness nodes
    int lblocks, tblocks;  // slow: secondary length and thickness blocks
    int off_r, off_t, off_phi, off_sl, off_slw, off_st, pad0, pad1;
};
static_assert(sizeof(ZAxisHeader) % 16 == 0, "z-axis header alignment");

bool buildZAxis(const Coil &prim, const Coil &sec, const PrecisionArgs &pz, const PrecisionArgs &sz,
                std::vector<unsigned char> &blob, std::string &err)
{
    if (!validArgs(pz) || !validArgs(sz))
    {
        err = "z-axis pair precision arguments out of range (increments 1..100, blocks >= 1)";
        return false;
    }
    ZAxisHeader z;
    std::memset(&z, 0, sizeof(z));
    const bool fastPrim = prim.coil_type == 0 || prim.coil_type == 1;
    const bool fastSec = sec.coil_type == 0 || sec.coil_type == 1;
    z.fast = fastPrim && fastSec ? 1 : 0;
    z.prim_length = prim.length;
    z.sec_length = sec.length;
    z.prim_current = prim.current;
    z.sec_current = sec.current;
    z.sec_turns = sec.num_turns;
    const int hdr16 = (int)sizeof(ZAxisHeader) / 16;
    std::vector<double> t0, t1, t2, t3, t4, t5;  // tables in blob order
    if (z.fast)
    {
        const double thicknessBlock = prim.thickness / pz.thickness_blocks;
        const double angularBlock = kPi / pz.angular_blocks;
        const double radialBlock = sec.thickness / sz.thickness_blocks;
        z.fast_constant = kMuReduced * prim.current_density * sec.current_density * thicknessBlock * angularBlock *
                          radialBlock * 0.125;
        const double *rx = legendreNodes(sz.thickness_increments), *rw = legendreWeights(sz.thickness_increments);
        for (int b = 0; b < sz.thickness_blocks; ++b)
        {
            const double blockPositionR = sec.inner_radius + radialBlock * (b + 0.5);
            for (int i = 0; i < sz.thickness_increments; ++i)
                t0.insert(t0.end(), {blockPositionR + (radialBlock * 0.5) * rx[i], rw[i]});
        }
        const double *tx = legendreNodes(pz.thickness_increments), *tw = legendreWeights(pz.thickness_increments);
        for (int b = 0; b < pz.thickness_blocks; ++b)
        {
            const double blockPositionT = prim.inner_radius + thicknessBlock * (b + 0.5);
            for (int i = 0; i < pz.thickness_increments; ++i)
                t1.insert(t1.end(), {blockPositionT + (thicknessBlock * 0.5) * tx[i], tw[i]});
        }
        const double *ax = legendreNodes(pz.angular_increments), *aw = legendreWeights(pz.angular_increments);
        for (int b = 0; b < pz.angular_blocks; ++b)
        {
            const double blockPositionPhi = angularBlock * (b + 0.5);
            for (int i = 0; i < pz.angular_increments; ++i)
                t2.insert(t2.end(), {std::cos(blockPositionPhi + (angularBlock * 0.5) * ax[i]), aw[i]});
        }
        z.n_r = (int)t0.size() / 2;
        z.n_t = (int)t1.size() / 2;
        z.n_phi = (int)t2.size() / 2;
        z.off_r = hdr16;
        z.off_t = z.off_r + z.n_r;
        z.off_phi = z.off_t + z.n_t;
    }
    else
    {
        // the primary's own field tables, then the secondary's (r, z) grid
        primaryTables(prim, pz, t0, t1, t2);
        SegmentHeader &h = z.prim;
        for (int i = 0; i < 3; ++i)
            h.position[i] = prim.position[i];
        std::memcpy(h.transform, prim.transform, sizeof(h.transform));
        std::memcpy(h.inv_transform, prim.inverse_transform, sizeof(h.inv_transform));
        h.half_length = prim.length * 0.5;
        h.field_factor = 1.0;
        h.inner_radius = prim.inner_radius;
        h.n_t = (int)t0.size() / 2;
        h.n_l = (int)t1.size() / 2;
        h.n_phi = (int)t2.size() / 2;
        h.fast = prim.use_fast_method != 0 ? 1 : 0;
        h.off_t = hdr16;
        h.off_l = h.off_t + h.n_t;
        h.off_phi = h.off_l + h.n_l;
        const double lengthBlockSize = sec.length / sz.length_blocks;
        const double thicknessBlockSize = sec.thickness / sz.thickness_blocks;
        const double *lx = legendreNodes(sz.length_increments), *lw = legendreWeights(sz.length_increments);
        for (int b = 0; b < sz.length_blocks; ++b)
        {
            const double zBlockPosition = (-1) * (sec.length * 0.5) + lengthBlockSize * (b + 0.5);
            for (int i = 0; i < sz.length_increments; ++i)
            {
                t3.insert(t3.end(), {zBlockPosition, (lengthBlockSize * 0.5) * lx[i]});
                t4.insert(t4.end(), {lw[i], 0.0});
            }
        }
        const double *tx = legendreNodes(sz.thickness_increments), *tw = legendreWeights(sz.thickness_increments);
        for (int b = 0; b < sz.thickness_blocks; ++b)
        {
            const double rBlockPosition = sec.inner_radius + thicknessBlockSize * (b + 0.5);
            for (int i = 0; i < sz.thickness_increments; ++i)
                t5.insert(t5.end(), {rBlockPosition + (thicknessBlockSize * 0.5) * tx[i], tw[i]});
        }
        z.n_sl = (int)t3.size() / 2;
        z.n_st = (int)t5.size() / 2;
        z.lblocks = sz.length_blocks;
        z.tblocks = sz.thickness_blocks;
        z.off_sl = h.off_phi + h.n_phi;
        z.off_slw = z.off_sl + z.n_sl;
        z.off_st = z.off_slw + z.n_sl;
    }
    put(blob, &z, sizeof(z));
    for (const std::vector<double> *t : {&t0, &t1, &t2, &t3, &t4, &t5})
        put(blob, t->data(), sizeof(double) * t->size());
    return true;
}

// Full warp: the z-axis value of one coaxial pair -- mutual inductance
// (QTY 0) or axial force on the secondary (QTY 1) -- for the primary at pose P
// and the secondary centre at z = secZ (every lane returns the same value)
template <int QTY>
__device__ double zAxisValue(const unsigned char *zb, const Pose &P, double secZ, int lane)
{
    const ZAxisHeader &z = *reinterpret_cast<const ZAxisHeader *>(zb);
    const double2 *base = reinterpret_cast<const double2 *>(zb);
    double part = 0.0;
    if (z.fast)
    {
        const double2 *rn = base + z.off_r, *tn = base + z.off_t, *pn = base + z.off_phi;
        const double zd = sub(secZ, P.pos[2]);
        const double hs = mul(z.sec_length, 0.5), hp = mul(z.prim_length, 0.5);
        const double z1 = add(add(zd, hs), hp), z2 = sub(add(zd, hs), hp);
        const double z3 = sub(sub(zd, hs), hp), z4 = add(sub(zd, hs), hp);
        const double z1s = mul(z1, z1), z2s = mul(z2, z2), z3s = mul(z3, z3), z4s = mul(z4, z4);
        const long long n = (long long)z.n_r * z.n_t * z.n_phi;
        for (long long e = lane; e < n; e += 32)
        {
            const int k = (int)(e % z.n_phi);
            const long long ij = e / z.n_phi;
            const int j = (int)(ij % z.n_t), i = (int)(ij / z.n_t);
            const double2 R = rn[i], T = tn[j], F = pn[k];
            const double tempConst = mul(mul(z.fast_constant, R.y), T.y);
            const double A = mul(mul(2.0, T.x), R.x);
            const double B = add(mul(T.x, T.x), mul(R.x, R.x));
            const double c = F.x;
            const double C = sub(B, mul(A, c));
            const double D = sqr(C);
            double term;
            if (QTY == 0)
            {
                const double E1 = sqr(add(C, z1s)), E2 = sqr(add(C, z2s));
                const double E3 = sqr(add(C, z3s)), E4 = sqr(add(C, z4s));
                const double F1 = dvd(z1, D), F2 = dvd(z2, D), F3 = dvd(z3, D), F4 = dvd(z4, D);
                const double G1 = sqr(add(mul(F1, F1), 1.0)), G2 = sqr(add(mul(F2, F2), 1.0));
                const double G3 = sqr(add(mul(F3, F3), 1.0)), G4 = sqr(add(mul(F4, F4), 1.0));
                const double H1 = mul(z1, log(add(F1, G1))), H2 = mul(z2, log(add(F2, G2)));
                const double H3 = mul(z3, log(add(F3, G3))), H4 = mul(z4, log(add(F4, G4)));
                const double S = add(sub(add(sub(sub(add(sub(H1, H2), H3), H4), E1), E2), E3), E4);
                term = mul(mul(mul(mul(tempConst, F.y), A), c), S);
            }
            else
            {
                const double E1 = dvd(z1, D), E2 = dvd(z2, D), E3 = dvd(z3, D), E4 = dvd(z4, D);
                const double G1 = add(E1, sqr(add(mul(E1, E1), 1.0))), G2 = add(E2, sqr(add(mul(E2, E2), 1.0)));
                const double G3 = add(E3, sqr(add(mul(E3, E3), 1.0))), G4 = add(E4, sqr(add(mul(E4, E4), 1.0)));
                const double H = log(dvd(mul(G2, G4), mul(G1, G3)));
                term = mul(mul(mul(mul(tempConst, F.y), A), c), H);
            }
            part += term;
        }
    }
    else
    {
        const SegmentHeader &h = z.prim;
        const double2 *tt = base + h.off_t, *lt = base + h.off_l, *pt = base + h.off_phi;
        const double2 *sl = base + z.off_sl, *slw = base + z.off_slw, *st = base + z.off_st;
        const int n = z.n_sl * z.n_st;
        for (int e = lane; e < n; e += 32)
        {
            const int l = e / z.n_st, t = e % z.n_st;
            const double2 L = sl[l], R = st[t];
            const double pz = add(add(secZ, L.x), L.y);
            const double w = mul(mul(mul(0.25, R.x), slw[l].x), R.y);
            const Frame f = toCoilFrameAt(P.pos, P.Ti, R.x, 0.0, pz);
            if (QTY == 0)
            {
                const double a = segmentA64<1>(h, tt, lt, pt, f, 0);
                const double vx = -a * f.sphi, vy = a * f.cphi;
                const double Ax = add(mul(P.T[0], vx), mul(P.T[1], vy));
                const double Ay = add(mul(P.T[3], vx), mul(P.T[4], vy));
                const double Az = add(mul(P.T[6], vx), mul(P.T[7], vy));
                part += mul(sqr(add(add(mul(Ax, Ax), mul(Ay, Ay)), mul(Az, Az))), w);
            }
            else
            {
                double H, Z;
                segmentB64<1>(h, tt, lt, pt, f, 0, H, Z);
                const double Bx = add(add(mul(P.T[0], mul(H, f.cphi)), mul(P.T[1], mul(H, f.sphi))), mul(P.T[2], Z));
                part += mul(Bx, w);
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off /= 2)
        part += __shfl_xor_sync(0xffffffffu, part, off);
    if (z.fast)
        return QTY == 0 ? dvd(mul(part, 2 * kPi), mul(z.prim_current, z.sec_current)) : mul(mul(-1.0, part), 2 * kPi);
    const double avg = dvd(part, (double)(z.lblocks * z.tblocks));
    return QTY == 0 ? dvd(mul(mul(avg, 2 * kPi), z.sec_turns), z.prim_current)
                    : mul(mul(mul(mul(-1.0, avg), 2 * kPi), z.sec_turns), z.sec_current);
}

// Second pass over the arrangements the general kernel recorded as having a
// coaxial primary: one warp per arrangement, primaries in order.
template <int QTY>
__global__ void __launch_bounds__(128) zAxisKernel(const unsigned char *__restrict__ blob,
                                                   const long long *__restrict__ primOffsets,
                                                   const long long *__restrict__ zOffsets, int nprim,
                                                   const double *__restrict__ primPoses,
                                                   const double *__restrict__ secPoses,
                                                   const long long *__restrict__ list,
                                                   const unsigned long long *__restrict__ listCount,
                                                   double *__restrict__ out)
{
    constexpr int W = QTY == 0 ? 1 : 6;
    const int lane = threadIdx.x % 32;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const long long warps = (long long)gridDim.x * blockDim.x / 32;
    const long long n = (long long)*listCount;
    for (long long e = warp; e < n; e += warps)
    {
        const long long a = list[e];
        const double *sp = secPoses + 5 * a;
        double total = 0.0;
        for (int j = 0; j < nprim; ++j)
        {
            if (zOffsets[j] < 0)
                continue;
            const PairHeader &ph = *reinterpret_cast<const PairHeader *>(blob + primOffsets[j]);
            const SegmentHeader &h = ph.prim;
            Pose P;
            double ppose[5];
            if (primPoses)
            {
                for (int i = 0; i < 5; ++i)
                    ppose[i] = primPoses[5 * a + i];
                poseFromAngles(ppose, P);
            }
            else
            {
                for (int i = 0; i < 3; ++i)
                    P.pos[i] = ppose[i] = h.position[i];
                for (int i = 0; i < 9; ++i)
                {
                    P.T[i] = h.transform[i];
                    P.Ti[i] = h.inv_transform[i];
                }
                ppose[3] = ph.prim_y_angle;
                ppose[4] = ph.prim_z_angle;
            }
            if (!zAxisCase(ppose, sp, h.inner_radius))
                continue;
            total += zAxisValue<QTY>(blob + zOffsets[j], P, sp[2], lane);
        }
        if (lane == 0)
            out[W * a + (QTY == 1 ? 2 : 0)] += total;
    }
}
