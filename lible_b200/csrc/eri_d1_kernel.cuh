// First nuclear derivatives of contracted shell quartets, one instantiation per class, following
// the structure of src/lible/ints/twoel/eri_kernel_funs.hpp:350-515:
//   d/dA = (a/p) E_ab dR/dP E_cd^T + E1_ab R E_cd^T,    d/dB = (b/p) E_ab dR/dP E_cd^T - E1_ab R E_cd^T,
//   d/dC = E_ab (-(c/q) dR/dP E_cd^T + R E1_cd^T),     d/dD = -(d/dA + d/dB + d/dC),
// where dR/dP_x is the R matrix shifted by one unit along x (Boys function to L+1) and E1 is the
// derivative of the Hermite coefficients with respect to the pair separation.
//
// Per primitive quartet the R recursion runs once (to L+1); from it the block gathers the three
// shifted R matrices and the plain one and forms the seven ket-side products
//   dR/dP_x E_cd^T (x = 0..2),  R E_cd^T,  R E1_cd,x^T (x = 0..2)
// into per-thread accumulators (four "passes": x, y, z and plain).  The bra-side contractions with
// E_ab and E1_ab follow once per bra primitive.  The ket E and E1 tiles of a primitive are staged in
// shared memory when the class's layout fits.  Two epilogues:
//   kD1Store: the 12 blocks are accumulated straight into the caller's output (each element owned
//             by exactly one thread, so no atomics);
//   kD1Grad:  each block is contracted on the fly with the two-particle density of
//             E = 1/2 Tr(DJ) - 1/4 Tr(DK),  Gamma = f (4 D_ab D_cd - D_ac D_bd - D_ad D_bc),
//             and the per-atom sums are added to the gradient (the adjoint of the J/K build);
//   kD1GradRI: the same for the RI-J energy E = 1/2 gamma^T (P|Q)^{-1} gamma, whose gradient is
//             sum_P d_P sum_mn D_mn d(mn|P) - 1/2 sum_PQ d_P d_Q d(P|Q) with d = (P|Q)^{-1} gamma:
//             Gamma = w D_mn d_P for three-centre blocks and -w/2 d_P d_Q for two-centre ones, w the
//             multiplicity of the unique pair (2, or 1 for a shell with itself).
#pragma once

#include "device_common.cuh"
#include "eri_kernel.cuh"  // DMMA fragment helpers and operand pitches

namespace lible_b200
{
    template <int LA, int LB, int LC, int LD>
    struct ShapeD1
    {
        using C = Cls<LA, LB, LC, LD>;
        static constexpr int HS = C::HAB * C::SCD;
        // at most 4 accumulator slots per thread and pass, up to 256 threads
        static constexpr int G0 = 32 * ((HS + 127) / 128);
        static constexpr int G = G0 < 32 ? 32 : (G0 > 256 ? 256 : G0);
        static constexpr int IK = (HS + G - 1) / G;
        static constexpr size_t off_rb = 0;                                        // 2 x NR1 doubles
        static constexpr size_t off_rm = off_rb + 8 * 2 * C::NR1;                  // HCD x HAB
        static constexpr size_t off_rx = off_rm + 8 * C::HCD * C::HAB;             // 2 x HAB x SCD
        static constexpr size_t off_gm = off_rx + 8 * 2 * C::HAB * C::SCD;         // SAB x SCD
        static constexpr size_t off_st = off_gm + 8 * C::SAB * C::SCD;             // HCD x HAB char4
        static constexpr size_t off_ht = off_st + 4 * C::HCD * C::HAB;             // NR1 char4
        static constexpr size_t off_rd = (off_ht + 4 * C::NR1 + 15) / 16 * 16;    // 9 x G/32 doubles
        static constexpr size_t off_ek = off_rd + 8 * 9 * (G / 32);                // 4 x HCD x SCD (staged)
        static constexpr size_t smem_stage = off_ek + 8 * 4 * C::HCD * C::SCD;
        static constexpr bool STAGE = smem_stage <= 200 * 1024;
        static constexpr size_t smem = STAGE ? smem_stage : off_ek;
    };

    template <int LA, int LB, int LC, int LD>
    __global__ void __launch_bounds__(ShapeD1<LA, LB, LC, LD>::G) eriD1Kernel(QuartetArgs a)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = ShapeD1<LA, LB, LC, LD>;
        constexpr int G = S::G;
        constexpr int L1 = C::L + 1;
        constexpr int blk = C::SAB * C::SCD;
        extern __shared__ __align__(16) unsigned char smem[];
        double *rb = reinterpret_cast<double *>(smem + S::off_rb);
        double *rm = reinterpret_cast<double *>(smem + S::off_rm);
        double *rx1 = reinterpret_cast<double *>(smem + S::off_rx);
        double *rx2 = rx1 + C::HAB * C::SCD;
        double *gm = reinterpret_cast<double *>(smem + S::off_gm);
        char4 *st = reinterpret_cast<char4 *>(smem + S::off_st);
        char4 *ht = reinterpret_cast<char4 *>(smem + S::off_ht);
        const int tid = threadIdx.x;

        for (int e = tid; e < C::NR1; e += G)
        {
            int t, u, v;
            hermTuv(e, t, u, v);
            ht[e] = make_char4((char)t, (char)u, (char)v, (char)(t + u + v));
        }
        for (int e = tid; e < C::HCD * C::HAB; e += G)
        {
            const int hp = e / C::HAB, h = e % C::HAB;
            int t, u, v, tp, up, vp;
            hermTuv(h, t, u, v);
            hermTuv(hp, tp, up, vp);
            st[e] = make_char4((char)(t + tp), (char)(u + up), (char)(v + vp), (char)((tp + up + vp) & 1));
        }
        __syncthreads();

        // one quartet at a time for the whole block
        auto processTask = [&](long long task, uint32_t ib, uint32_t ik) {
            const int32_t *bi = a.bra.info + 8 * ib;
            const int32_t *ki = a.ket.info + 8 * ik;
            double acc[12];
#pragma unroll
            for (int x = 0; x < 12; x++)
                acc[x] = 0.0;
            double *outq = nullptr;
            if (a.mode == kD1Store)
            {
                outq = a.out + (size_t)task * 12 * blk;
                for (int e = tid; e < 12 * blk; e += G)
                    outq[e] = 0.0;
            }
            else if (a.mode == kD1GradRI)
            {
                const int n = a.nao;
                if (a.aux_side == 2)
                {
                    const double w = (a.same_class && ib == ik) ? 0.5 : 1.0;  // -w/2 with w = 1 or 2
                    for (int e = tid; e < blk; e += G)
                    {
                        const int P = bi[0] + e / C::SCD, Q = ki[0] + e % C::SCD;
                        gm[e] = -w * a.dcoef[P] * a.dcoef[Q];
                    }
                }
                else
                {
                    const int32_t *mi = a.aux_side == 0 ? bi : ki;
                    const double w = mi[4] == mi[5] ? 1.0 : 2.0;
                    for (int e = tid; e < blk; e += G)
                    {
                        const int mn = e / C::SCD, kt = e % C::SCD;
                        int mu, nu, P;
                        if (a.aux_side == 0)
                        {
                            mu = bi[0] + mn / C::SB;
                            nu = bi[1] + mn % C::SB;
                            P = ki[0] + kt;
                        }
                        else
                        {
                            P = bi[0] + mn;
                            mu = ki[0] + kt / C::SD;
                            nu = ki[1] + kt % C::SD;
                        }
                        gm[e] = w * a.D[(size_t)mu * n + nu] * a.dcoef[P];
                    }
                }
            }
            else
            {
                const double f = quartetWeight(a, ib, ik);
                const int n = a.nao;
                for (int e = tid; e < blk; e += G)
                {
                    const int mn = e / C::SCD, kt = e % C::SCD;
                    const int mu = bi[0] + mn / C::SB, nu = bi[1] + mn % C::SB;
                    const int ka = ki[0] + kt / C::SD, ta = ki[1] + kt % C::SD;
                    const double *D = a.D;
                    gm[e] = f * (4.0 * D[(size_t)mu * n + nu] * D[(size_t)ka * n + ta] -
                                 D[(size_t)mu * n + ka] * D[(size_t)nu * n + ta] -
                                 D[(size_t)mu * n + ta] * D[(size_t)nu * n + ka]);
                }
            }
            __syncthreads();

            // Output slot of internal block (centre c, direction x) for kD1Store.
            auto emit = [&](int centre, int x, int e, double v) {
                if (a.mode == kD1Store)
                    outq[(size_t)(centre * 3 + x) * blk + e] += v;
                else
                    acc[centre * 3 + x] += gm[e] * v;
            };

            const uint32_t p0 = a.bra.pofs[ib], p1 = a.bra.pofs[ib + 1];
            const uint32_t q0 = a.ket.pofs[ik], q1 = a.ket.pofs[ik + 1];
            for (uint32_t p = p0; p < p1; p++)
            {
                const PQ4 P = loadPQ(a.bra.pP, p);
                const double2 AB = __ldg(reinterpret_cast<const double2 *>(a.bra.ab) + p);
                const double *eab = a.bra.E + (size_t)p * C::SAB * C::HAB;
                const double *e1ab = a.bra.E1 + (size_t)p * 3 * C::SAB * C::HAB;
                // r1[x]: dR/dP_x E_cd^T (x < 3) and R E_cd^T (x = 3);
                // r2[x]: -(c/q) dR/dP_x E_cd^T + R E1_cd,x^T.  Classes with at most 4 accumulator
                // slots per thread keep all four passes live and sweep the ket primitives once; larger
                // ones sweep once per pass (NPG = 1) to bound the live state.
                constexpr int NPG = S::IK <= 4 ? 4 : 1;
                for (int pg = 0; pg < 4; pg += NPG)
                {
                double r1[NPG][S::IK], r2[NPG][S::IK];
#pragma unroll
                for (int k = 0; k < S::IK; k++)
#pragma unroll
                    for (int x = 0; x < NPG; x++)
                        r1[x][k] = r2[x][k] = 0.0;
                for (uint32_t q = q0; q < q1; q++)
                {
                    const PQ4 Q = loadPQ(a.ket.pP, q);
                    const double cexp = __ldg(a.ket.ab + 2 * q);
                    const double rs = rsqrt(P.x + Q.x);
                    const double alpha = P.x * Q.x * (rs * rs);
                    const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                    const double fac = 34.986836655249725 * rs * P.ip * Q.ip;
                    double F[L1 + 1];
                    boysF<L1, false>(alpha * (X * X + Y * Y + Z * Z), a.boys + L1 * kBoysTerms * kBoysPitch, F);
                    const double m2a = -2.0 * alpha;
                    double *cur = rb, *nxt = rb + C::NR1;
                    if (!closedFormR<L1>() && tid == 0)
                    {
                        double pw = 1.0;
                        for (int k = 0; k < L1; k++)
                            pw *= m2a;
                        cur[0] = F[L1] * fac * pw;
                    }
                    // ket E and E1 tiles of this primitive (staged when the layout fits)
                    const double *ecd = a.ket.Et + (size_t)q * C::HCD * C::SCD;
                    const double *e1cd = a.ket.E1t + (size_t)q * 3 * C::HCD * C::SCD;
                    if constexpr (S::STAGE)
                    {
                        // copies land during the R build; waited for before the first product
                        double *ek = reinterpret_cast<double *>(smem + S::off_ek);
                        for (int e = tid; e < C::HCD * C::SCD; e += G)
                            cpAsync8(ek + e, ecd + e);
                        for (int e = tid; e < 3 * C::HCD * C::SCD; e += G)
                            cpAsync8(ek + C::HCD * C::SCD + e, e1cd + e);
                        ecd = ek;
                        e1cd = ek + C::HCD * C::SCD;
                    }
                    if constexpr (closedFormR<L1>())
                    {
                        groupHermiteR<L1, double>(F, fac, m2a, X, Y, Z, nxt, cur, ht, tid, G);
                    }
                    else
                    {
                    __syncthreads();
#pragma unroll
                    for (int n = L1 - 1; n >= 0; n--)
                    {
                        const int cnt = nherm(L1 - n);
                        for (int e = tid; e < cnt; e += G)
                        {
                            double r;
                            if (e == 0)
                            {
                                double pn = 1.0;
                                for (int k = 0; k < n; k++)
                                    pn *= m2a;
                                r = F[n] * fac * pn;
                            }
                            else
                            {
                                const char4 tv = ht[e];
                                const int t = tv.x, u = tv.y, v = tv.z, m = tv.w;
                                if (t > 0)
                                {
                                    r = X * cur[nherm(m - 2) + cartIndex(u, v)];
                                    if (t > 1)
                                        r += (t - 1) * cur[nherm(m - 3) + cartIndex(u, v)];
                                }
                                else if (u > 0)
                                {
                                    r = Y * cur[nherm(m - 2) + cartIndex(u - 1, v)];
                                    if (u > 1)
                                        r += (u - 1) * cur[nherm(m - 3) + cartIndex(u - 2, v)];
                                }
                                else
                                {
                                    r = Z * cur[nherm(m - 2) + cartIndex(0, v - 1)];
                                    if (v > 1)
                                        r += (v - 1) * cur[nherm(m - 3) + cartIndex(0, v - 2)];
                                }
                            }
                            nxt[e] = r;
                        }
                        __syncthreads();
                        double *tmp = cur;
                        cur = nxt;
                        nxt = tmp;
                    }
                    }
                    const double cq = cexp / Q.x;
                    // shifted R (passes x, y, z) and plain R (pass 3, and the E1_cd terms of the
                    // x, y, z passes) from the one recursion
#pragma unroll
                    for (int j = 0; j < NPG; j++)
                    {
                        const int pass = pg + j;
                        const int dx = pass == 0, dy = pass == 1, dz = pass == 2;
                        for (int e = tid; e < C::HCD * C::HAB; e += G)
                        {
                            const char4 s4 = st[e];
                            const double r = cur[hermIndex(s4.x + dx, s4.y + dy, s4.z + dz)];
                            rm[e] = s4.w ? -r : r;
                        }
                        if constexpr (S::STAGE)
                            cpAsyncWaitAll();  // the staged ket tiles (no-op after the first pass)
                        __syncthreads();
#pragma unroll
                        for (int k = 0; k < S::IK; k++)
                        {
                            const int e = tid + G * k;
                            if (e < C::HAB * C::SCD)
                            {
                                const int h = e / C::SCD, c = e % C::SCD;
                                double sv = 0.0;
                                for (int hp = 0; hp < C::HCD; hp++)
                                    sv += rm[hp * C::HAB + h] * ecd[hp * C::SCD + c];
                                r1[j][k] += sv;
                                if (pass < 3)
                                    r2[j][k] -= cq * sv;
                                else if constexpr (NPG == 4)
                                {
#pragma unroll
                                    for (int x = 0; x < 3; x++)
                                    {
                                        const double *e1 = e1cd + x * C::HCD * C::SCD;
                                        double s1 = 0.0;
                                        for (int hp = 0; hp < C::HCD; hp++)
                                            s1 += rm[hp * C::HAB + h] * e1[hp * C::SCD + c];
                                        r2[x][k] += s1;
                                    }
                                }
                            }
                        }
                        __syncthreads();
                        if constexpr (NPG == 1)
                        {
                            if (pass < 3)
                            {
                                // this pass's E1_cd term needs the plain R matrix
                                for (int e = tid; e < C::HCD * C::HAB; e += G)
                                {
                                    const char4 s4 = st[e];
                                    const double r = cur[hermIndex(s4.x, s4.y, s4.z)];
                                    rm[e] = s4.w ? -r : r;
                                }
                                __syncthreads();
                                const double *e1 = e1cd + pass * C::HCD * C::SCD;
#pragma unroll
                                for (int k = 0; k < S::IK; k++)
                                {
                                    const int e = tid + G * k;
                                    if (e < C::HAB * C::SCD)
                                    {
                                        const int h = e / C::SCD, c = e % C::SCD;
                                        double s1 = 0.0;
                                        for (int hp = 0; hp < C::HCD; hp++)
                                            s1 += rm[hp * C::HAB + h] * e1[hp * C::SCD + c];
                                        r2[j][k] += s1;
                                    }
                                }
                                __syncthreads();
                            }
                        }
                    }
                }
                // bra side of the passes of this group
#pragma unroll
                for (int j = 0; j < NPG; j++)
                {
                    const int pass = pg + j;
#pragma unroll
                    for (int k = 0; k < S::IK; k++)
                    {
                        const int e = tid + G * k;
                        if (e < C::HAB * C::SCD)
                        {
                            rx1[e] = r1[j][k];
                            if (pass < 3)
                                rx2[e] = NPG == 4 ? r2[pass][k] : r2[j][k];
                        }
                    }
                    __syncthreads();
                    for (int e = tid; e < blk; e += G)
                    {
                        const int m = e / C::SCD, c = e % C::SCD;
                        if (pass < 3)
                        {
                            double sp = 0.0, sc = 0.0;
                            for (int h = 0; h < C::HAB; h++)
                            {
                                const double ev = eab[m * C::HAB + h];
                                sp += ev * rx1[h * C::SCD + c];
                                sc += ev * rx2[h * C::SCD + c];
                            }
                            emit(0, pass, e, (AB.x / P.x) * sp);
                            emit(1, pass, e, (AB.y / P.x) * sp);
                            emit(2, pass, e, sc);
                        }
                        else
                        {
                            for (int x = 0; x < 3; x++)
                            {
                                double sv = 0.0;
                                for (int h = 0; h < C::HAB; h++)
                                    sv += e1ab[(x * C::SAB + m) * C::HAB + h] * rx1[h * C::SCD + c];
                                emit(0, x, e, sv);
                                emit(1, x, e, -sv);
                            }
                        }
                    }
                    __syncthreads();
                }
                }
            }

            if (a.mode == kD1Store)
            {
                // D by translational invariance; the caller's orientation is applied afterwards by
                // a separate reorder pass
                for (int e = tid; e < blk; e += G)
                    for (int x = 0; x < 3; x++)
                        outq[(size_t)(9 + x) * blk + e] =
                            -(outq[(size_t)x * blk + e] + outq[(size_t)(3 + x) * blk + e] + outq[(size_t)(6 + x) * blk + e]);
            }
            else
            {
                // reduce the 9 independent sums over the block, then add per atom
                double *red = reinterpret_cast<double *>(smem + S::off_rd);
                for (int x = 0; x < 9; x++)
                {
                    double v = acc[x];
                    for (int o = 16; o > 0; o >>= 1)
                        v += __shfl_down_sync(0xffffffffu, v, o);
                    if ((tid & 31) == 0)
                        red[(tid >> 5) * 9 + x] = v;
                }
                __syncthreads();
                if (tid < 9)
                {
                    double v = 0.0;
                    for (int w = 0; w < G / 32; w++)
                        v += red[w * 9 + tid];
                    const int centre = tid / 3, x = tid % 3;
                    const int atom = centre == 0 ? bi[2] : centre == 1 ? bi[3] : ki[2];
                    atomicAdd(a.grad + 3 * atom + x, v);
                    atomicAdd(a.grad + 3 * ki[3] + x, -v);
                }
                __syncthreads();
            }
        };

        // the block's tasks come in increasing order, so one forward-moving cursor decodes them
        // (a load or two per task instead of a binary search)
        int cur = 0;
        auto runTask = [&](long long task) {
            uint32_t ib, ik;
            decodeCursor(a, task, cur, ib, ik);
            if (inWindow(a, ib, ik, 0, false))
                processTask(task, ib, ik);
        };
        if (a.chunks)
        {
            // work queue: the block claims chunks of consecutive tasks
            __shared__ unsigned long long claimed;
            for (;;)
            {
                if (tid == 0)
                    claimed = atomicAdd(a.counter, 1ULL);
                __syncthreads();
                const unsigned long long c = claimed;
                __syncthreads();
                if (c >= (unsigned long long)a.n_chunks)
                    break;
                const long long t1 = (long long)__ldg(a.chunks + c + 1);
                for (long long t = (long long)__ldg(a.chunks + c); t < t1; t++)
                    runTask(t);
            }
        }
        else
            for (long long task = blockIdx.x; task < a.n_tasks; task += gridDim.x)
                runTask(task);
    }

    // ---------------------------------------------------------------------------------------
    // Register form of the gradient contraction (J/K, kD1Grad, and RI-J, kD1GradRI) for the classes
    // of d1RegisterClass: GT threads per quartet, each owning S_cd / GT ket columns.  With Gamma the
    // density block of the quartet (as in the block kernel's epilogues) and, per bra primitive,
    // GE = Gamma^T E_ab and GE1_x = Gamma^T E1_ab,x, the gradient terms of the formulas above become
    // per primitive quartet
    //   t1_x  = sum GE  . (dR/dP_x E_cd^T),   t13_x = sum GE1_x . (R E_cd^T),
    //   tc_x  = sum GE  . (-(c/q) dR/dP_x E_cd^T + R E1_cd,x^T),
    // and A_x += (a/p) t1_x + t13_x, B_x += (b/p) t1_x - t13_x, C_x += tc_x (D by invariance).
    template <int LA, int LB, int LC, int LD>
    __device__ __forceinline__ void quartetD1Reg(const QuartetArgs &a, uint32_t ib, uint32_t ik, int c0, double *g)
    {
        using C = Cls<LA, LB, LC, LD>;
        constexpr int L1 = C::L + 1;
        // this thread's ket columns [c0, c0 + CW)
        constexpr int CW = C::SCD / d1RegisterGroup(LA, LB, LC, LD);
        const int32_t *bi = a.bra.info + 8 * ib;
        const int32_t *ki = a.ket.info + 8 * ik;
        const size_t n = (size_t)a.nao;
        const double *D = a.D;
        double gam[C::SAB * CW];
        if (a.mode == kD1GradRI)
        {
            // RI-J: w D_mn d_P (three-centre, the auxiliary shell on either side) or -w/2 d_P d_Q
            // (two-centre), w the multiplicity of the unique pair, as in the block kernel
            const int32_t *mi = a.aux_side == 0 ? bi : ki;
            const double w = a.aux_side == 2 ? -((a.same_class && ib == ik) ? 0.5 : 1.0) : (mi[4] == mi[5] ? 1.0 : 2.0);
#pragma unroll
            for (int m = 0; m < C::SAB; m++)
#pragma unroll
                for (int cw = 0; cw < CW; cw++)
                {
                    const int c = c0 + cw;
                    double v;
                    if (a.aux_side == 2)
                        v = __ldg(a.dcoef + bi[0] + m) * __ldg(a.dcoef + ki[0] + c);
                    else if (a.aux_side == 0)
                        v = __ldg(D + (size_t)(bi[0] + m / C::SB) * n + bi[1] + m % C::SB) * __ldg(a.dcoef + ki[0] + c);
                    else
                        v = __ldg(D + (size_t)(ki[0] + c / C::SD) * n + ki[1] + c % C::SD) * __ldg(a.dcoef + bi[0] + m);
                    gam[m * CW + cw] = w * v;
                }
        }
        else
        {
            const double f = quartetWeight(a, ib, ik);
#pragma unroll
            for (int m = 0; m < C::SAB; m++)
#pragma unroll
                for (int cw = 0; cw < CW; cw++)
                {
                    const int c = c0 + cw;
                    const size_t mu = bi[0] + m / C::SB, nu = bi[1] + m % C::SB;
                    const size_t ka = ki[0] + c / C::SD, ta = ki[1] + c % C::SD;
                    gam[m * CW + cw] = f * (4.0 * __ldg(D + mu * n + nu) * __ldg(D + ka * n + ta) -
                                               __ldg(D + mu * n + ka) * __ldg(D + nu * n + ta) -
                                               __ldg(D + mu * n + ta) * __ldg(D + nu * n + ka));
                }
        }
#pragma unroll
        for (int x = 0; x < 9; x++)
            g[x] = 0.0;
        const uint32_t p0 = a.bra.pofs[ib], p1 = a.bra.pofs[ib + 1];
        const uint32_t q0 = a.ket.pofs[ik], q1 = a.ket.pofs[ik + 1];
        for (uint32_t p = p0; p < p1; p++)
        {
            const PQ4 P = loadPQ(a.bra.pP, p);
            const double2 AB = __ldg(reinterpret_cast<const double2 *>(a.bra.ab) + p);
            const double *eab = a.bra.E + (size_t)p * C::SAB * C::HAB;
            const double *e1ab = a.bra.E1 + (size_t)p * 3 * C::SAB * C::HAB;
            double ge[C::HAB * CW], ge1[3 * C::HAB * CW];
#pragma unroll
            for (int h = 0; h < C::HAB; h++)
#pragma unroll
                for (int cw = 0; cw < CW; cw++)
                {
                    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
                    for (int m = 0; m < C::SAB; m++)
                    {
                        const double gm = gam[m * CW + cw];
                        s0 += gm * __ldg(eab + m * C::HAB + h);
                        s1 += gm * __ldg(e1ab + (0 * C::SAB + m) * C::HAB + h);
                        s2 += gm * __ldg(e1ab + (1 * C::SAB + m) * C::HAB + h);
                        s3 += gm * __ldg(e1ab + (2 * C::SAB + m) * C::HAB + h);
                    }
                    ge[h * CW + cw] = s0;
                    ge1[(0 * C::HAB + h) * CW + cw] = s1;
                    ge1[(1 * C::HAB + h) * CW + cw] = s2;
                    ge1[(2 * C::HAB + h) * CW + cw] = s3;
                }
            double t1[3] = {0, 0, 0}, t13[3] = {0, 0, 0}, tc[3] = {0, 0, 0};
            for (uint32_t q = q0; q < q1; q++)
            {
                const PQ4 Q = loadPQ(a.ket.pP, q);
                const double cq = __ldg(a.ket.ab + 2 * q) / Q.x;
                const double rs = rsqrt(P.x + Q.x);
                const double alpha = P.x * Q.x * (rs * rs);
                const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                const double fac = 34.986836655249725 * rs * P.ip * Q.ip;
                double F[L1 + 1];
                boysF<L1, false>(alpha * (X * X + Y * Y + Z * Z), a.boys + L1 * kBoysTerms * kBoysPitch, F);
#pragma unroll
                for (int k = 0; k <= L1; k++)
                    F[k] *= fac;
                double R[nherm(L1)];
                hermiteR<L1, double>(-2.0 * alpha, F, X, Y, Z, R);
                const double *ecd = a.ket.Et + (size_t)q * C::HCD * C::SCD;
                const double *e1cd = a.ket.E1t + (size_t)q * 3 * C::HCD * C::SCD;
#pragma unroll
                for (int h = 0, nh = 0; nh <= C::LAB; nh++)
#pragma unroll
                    for (int th = nh; th >= 0; th--)
#pragma unroll
                        for (int uh = nh - th; uh >= 0; uh--, h++)
                        {
                            const int vh = nh - th - uh;
#pragma unroll
                            for (int cw = 0; cw < CW; cw++)
                            {
                                const int c = c0 + cw;
                                double u0 = 0.0, ux = 0.0, uy = 0.0, uz = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
#pragma unroll
                                for (int hp = 0, np = 0; np <= C::LCD; np++)
#pragma unroll
                                    for (int tp = np; tp >= 0; tp--)
#pragma unroll
                                        for (int up = np - tp; up >= 0; up--, hp++)
                                        {
                                            const int vp = np - tp - up;
                                            const double sgn = (np & 1) ? -1.0 : 1.0;
                                            const double e0 = sgn * __ldg(ecd + hp * C::SCD + c);
                                            const int t = th + tp, u = uh + up, v = vh + vp;
                                            const double r0 = R[hermIndex(t, u, v)];
                                            u0 += r0 * e0;
                                            ux += R[hermIndex(t + 1, u, v)] * e0;
                                            uy += R[hermIndex(t, u + 1, v)] * e0;
                                            uz += R[hermIndex(t, u, v + 1)] * e0;
                                            const double rs0 = sgn * r0;
                                            vx += rs0 * __ldg(e1cd + (0 * C::HCD + hp) * C::SCD + c);
                                            vy += rs0 * __ldg(e1cd + (1 * C::HCD + hp) * C::SCD + c);
                                            vz += rs0 * __ldg(e1cd + (2 * C::HCD + hp) * C::SCD + c);
                                        }
                                const double gev = ge[h * CW + cw];
                                t1[0] += gev * ux;
                                t1[1] += gev * uy;
                                t1[2] += gev * uz;
                                t13[0] += ge1[(0 * C::HAB + h) * CW + cw] * u0;
                                t13[1] += ge1[(1 * C::HAB + h) * CW + cw] * u0;
                                t13[2] += ge1[(2 * C::HAB + h) * CW + cw] * u0;
                                tc[0] += gev * (vx - cq * ux);
                                tc[1] += gev * (vy - cq * uy);
                                tc[2] += gev * (vz - cq * uz);
                            }
                        }
            }
            const double ap = AB.x * P.ip, bp = AB.y * P.ip;
#pragma unroll
            for (int x = 0; x < 3; x++)
            {
                g[x] += ap * t1[x] + t13[x];
                g[3 + x] += bp * t1[x] - t13[x];
                g[6 + x] += tc[x];
            }
        }
    }

    // J/K-gradient kernel of the register classes: warps take 32 consecutive tasks of a work-queue
    // chunk (one per lane); each block sums its gradient in shared memory ([n_atoms][3], shared
    // atomics; the ket-centre terms of a warp whose lanes share the ket pair are summed by shuffles
    // first) and adds it to the output once.
    template <int LA, int LB, int LC, int LD>
    __global__ void __launch_bounds__(128) eriD1RegKernel(QuartetArgs a)
    {
        extern __shared__ __align__(16) double sg[];
        for (int e = threadIdx.x; e < 3 * a.n_atoms; e += blockDim.x)
            sg[e] = 0.0;
        __syncthreads();
        const int lane = threadIdx.x & 31;
        // GT threads per quartet (each owning S_cd / GT ket columns), QPW quartets per warp step
        constexpr int GT = d1RegisterGroup(LA, LB, LC, LD), QPW = 32 / GT;
        constexpr int CW = Cls<LA, LB, LC, LD>::SCD / GT;
        constexpr unsigned used = QPW * GT == 32 ? 0xffffffffu : ((1u << (QPW * GT)) - 1u);
        const int slot = lane / GT, member = lane % GT;
        // the task cursor carries over between the warp's chunks (increasing task order)
        int cur = 0;
        auto processRange = [&](long long start, long long end) {
            if (!a.list)
                cur = advanceMajor(a, start, cur);
            for (long long base = start; base < end; base += QPW)
            {
                const long long t = base + slot;
                uint32_t ib = 0, ik = 0;
                bool active = false;
                double g[9];
#pragma unroll
                for (int x = 0; x < 9; x++)
                    g[x] = 0.0;
                if (slot < QPW && t < end)
                {
                    int my = cur;
                    decodeCursor(a, t, my, ib, ik);
                    active = inWindow(a, ib, ik, 0, false);
                    if (active)
                        quartetD1Reg<LA, LB, LC, LD>(a, ib, ik, member * CW, g);
                }
                if (!a.list)
                    cur = advanceMajor(a, base + QPW < end ? base + QPW : end - 1, cur);
                const int32_t *bi = a.bra.info + 8 * ib;
                const int32_t *ki = a.ket.info + 8 * ik;
                // every used lane holds a quartet of one ket pair: the ket-centre terms are summed
                // across the warp (the group members' partial sums included)
                const unsigned vmask = __ballot_sync(0xffffffffu, active);
                const uint32_t ik0 = __shfl_sync(0xffffffffu, ik, 0);
                const bool uniform = vmask == used && __all_sync(0xffffffffu, !((used >> lane) & 1u) || ik == ik0);
#pragma unroll
                for (int x = 0; x < 3; x++)
                {
                    double gc = g[6 + x], gd = -(g[x] + g[3 + x] + g[6 + x]);
                    if (uniform)
                    {
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1)
                        {
                            gc += __shfl_xor_sync(0xffffffffu, gc, o);
                            gd += __shfl_xor_sync(0xffffffffu, gd, o);
                        }
                        if (lane == 0)
                        {
                            atomicAdd(sg + 3 * ki[2] + x, gc);
                            atomicAdd(sg + 3 * ki[3] + x, gd);
                        }
                    }
                    else if (active)
                    {
                        atomicAdd(sg + 3 * ki[2] + x, gc);
                        atomicAdd(sg + 3 * ki[3] + x, gd);
                    }
                    if (active)
                    {
                        atomicAdd(sg + 3 * bi[2] + x, g[x]);
                        atomicAdd(sg + 3 * bi[3] + x, g[3 + x]);
                    }
                }
            }
        };
        if (a.chunks)
        {
            for (;;)
            {
                unsigned long long c = 0;
                if (lane == 0)
                    c = atomicAdd(a.counter, 1ULL);
                c = __shfl_sync(0xffffffffu, c, 0);
                if (c >= (unsigned long long)a.n_chunks)
                    break;
                processRange((long long)__ldg(a.chunks + c), (long long)__ldg(a.chunks + c + 1));
            }
        }
        else
        {
            const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
            const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
            constexpr long long CH = 8 * 32;
            const long long n_chunks = (a.n_tasks + CH - 1) / CH;
            for (long long chunk = gw; chunk < n_chunks; chunk += warps)
                processRange(chunk * CH, (chunk + 1) * CH < a.n_tasks ? (chunk + 1) * CH : a.n_tasks);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * a.n_atoms; e += blockDim.x)
            if (sg[e] != 0.0)
                atomicAdd(a.grad + e, sg[e]);
    }

    // ---------------------------------------------------------------------------------------
    // Tensor-pipe form of the gradient contraction (kD1Grad, kD1GradRI) for the classes that are
    // not register classes.  With GE = Gamma^T E_ab and GE1_x = Gamma^T E1_ab,x formed once per bra
    // primitive, the seven ket-side products of a primitive quartet become traces
    //   W0 = GE E_cd^T,  W1_x = GE1_x E_cd^T,  W2_x = GE E1_cd,x^T   ([H_ab x H_cd], K = S_cd)
    //   t1_x  += sum_{h h'} W0[h][h'] s(h') R[h + h' + e_x],   t13_x += sum W1_x[h][h'] s(h') R[h + h'],
    //   tc_x  += sum W2_x[h][h'] s(h') R[h + h'] - (c/q) sum W0[h][h'] s(h') R[h + h' + e_x]
    // (s(h') = (-1)^{|h'|}, the terms of the register form above), so both the GE products
    // (H_ab x S_cd, K = S_ab) and the W products run as mma.m8n8k4.f64 tiles on the DMMA pipe.  The
    // accumulators of a W tile are consumed in registers: every lane gathers the R entries of its
    // own two elements.  One block (WD warps) per quartet; R by the shared recursion to L + 1.
    template <int LA, int LB, int LC, int LD>
    struct ShapeD1M
    {
        using C = Cls<LA, LB, LC, LD>;
        static constexpr int MT = (C::HAB + 7) / 8;                          // rows h of GE and W
        static constexpr int NT1 = (C::SCD + 7) / 8, KT1 = (C::SAB + 3) / 4;  // GE: N = c, K = m
        static constexpr int NT2 = (C::HCD + 7) / 8, KT2 = (C::SCD + 3) / 4;  // W: N = h', K = c
        static constexpr int TILES1 = MT * NT1, TILES2 = MT * NT2;
        static constexpr int WD0 = (TILES2 + 3) / 4;
        static constexpr int WD = WD0 < 2 ? 2 : (WD0 > 8 ? 8 : WD0);
        static constexpr int G = 32 * WD;
        // operand tiles: E_ab staged [m][h] (A^T of the GE product, k-major), Gamma [m][c] (k-major
        // B), GE [h][c] and E_cd [h'][c] (m-major A and B of the W product)
        static constexpr int P_EA = kPitch(MT * 8), P_G = kPitch(NT1 * 8);
        static constexpr int P_GE = mPitch(NT1 * 8 > KT2 * 4 ? NT1 * 8 : KT2 * 4), P_EC = mPitch(KT2 * 4);
        static constexpr size_t a16(size_t x) { return (x + 15) / 16 * 16; }
        static constexpr size_t off_rb = 0;                                               // 2 x NR1
        static constexpr size_t off_ea = a16(off_rb + 8 * 2 * C::NR1);                    // KT1*4 x P_EA
        static constexpr size_t off_g = a16(off_ea + 8 * (size_t)KT1 * 4 * P_EA);        // KT1*4 x P_G
        static constexpr size_t off_ge = a16(off_g + 8 * (size_t)KT1 * 4 * P_G);         // 4 x MT*8 x P_GE
        static constexpr size_t off_ec = a16(off_ge + 8 * 4 * (size_t)MT * 8 * P_GE);     // 4 x NT2*8 x P_EC
        static constexpr size_t off_rd = a16(off_ec + 8 * 4 * (size_t)NT2 * 8 * P_EC);    // 9 x WD
        static constexpr size_t off_ht = a16(off_rd + 8 * 9 * WD);                        // NR1 char4
        static constexpr size_t off_hab = a16(off_ht + 4 * C::NR1);                       // HAB char4
        static constexpr size_t off_hcd = a16(off_hab + 4 * C::HAB);                      // HCD char4
        static constexpr size_t smem1 = a16(off_hcd + 4 * C::HCD);
        // a second E_ab buffer (double buffering of the four E matrices of a bra primitive), kept
        // when it costs no resident block per SM (228 KB per SM, 1 KB reserved per block)
        static constexpr size_t off_ea2 = smem1;
        static constexpr size_t smem2 = a16(off_ea2 + 8 * (size_t)KT1 * 4 * P_EA);
        static constexpr size_t perSM(size_t x) { return (228 * 1024) / (x + 1024); }
        static constexpr bool DB = smem2 <= 200 * 1024 && perSM(smem2) >= perSM(smem1);
        static constexpr size_t smem = DB ? smem2 : smem1;
        // resident blocks per SM the register allocation must allow: as many as the shared memory
        // admits, at no fewer than 128 registers per thread
        static constexpr int MINB0 = (int)perSM(smem) < 65536 / (G * 128) ? (int)perSM(smem) : 65536 / (G * 128);
        static constexpr int MINB = MINB0 < 1 ? 1 : MINB0;
        // the classes this form serves, as measured on the (H2O)_8 cc-pVTZ gradient: not a register
        // class, a ket of at least S_cd = 5 spherical and H_cd = 10 Hermite functions (with smaller
        // kets the W products are too thin to pay for the GE products and the staging; (dd|ss), (fp|ss)
        // and (dd|ps) ran up to 2.3x slower than in the block form), and a layout that fits one block
        // per SM
        static constexpr bool USE = !d1RegisterClass(LA, LB, LC, LD) && C::SCD >= 5 && C::HCD >= 10 &&
                                    smem1 <= 200 * 1024;
    };

    template <int LA, int LB, int LC, int LD>
    __global__ void __launch_bounds__(ShapeD1M<LA, LB, LC, LD>::G, ShapeD1M<LA, LB, LC, LD>::MINB)
    eriD1MmaKernel(QuartetArgs a)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = ShapeD1M<LA, LB, LC, LD>;
        constexpr int G = S::G, WD = S::WD;
        constexpr int L1 = C::L + 1;
        extern __shared__ __align__(16) unsigned char smem[];
        double *rb = reinterpret_cast<double *>(smem + S::off_rb);
        double *ea = reinterpret_cast<double *>(smem + S::off_ea);
        double *gs = reinterpret_cast<double *>(smem + S::off_g);
        double *ge = reinterpret_cast<double *>(smem + S::off_ge);
        double *ec = reinterpret_cast<double *>(smem + S::off_ec);
        double *red = reinterpret_cast<double *>(smem + S::off_rd);
        char4 *ht = reinterpret_cast<char4 *>(smem + S::off_ht);
        char4 *hab = reinterpret_cast<char4 *>(smem + S::off_hab);
        char4 *hcd = reinterpret_cast<char4 *>(smem + S::off_hcd);
        const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, r8 = lane >> 2, k4 = lane & 3;
        constexpr size_t GE_SZ = (size_t)S::MT * 8 * S::P_GE, EC_SZ = (size_t)S::NT2 * 8 * S::P_EC;

        double *ea2 = reinterpret_cast<double *>(smem + S::off_ea2);  // second E_ab buffer (S::DB)
        // once per block: zero every operand tile (padding rows and columns are never written
        // afterwards, so they stay zero) and the Hermite (t, u, v, order) tables
        {
            const int nz = (int)((S::off_rd - S::off_ea) / 8);
            for (int e = tid; e < nz; e += G)
                ea[e] = 0.0;
            if constexpr (S::DB)
                for (int e = tid; e < S::KT1 * 4 * S::P_EA; e += G)
                    ea2[e] = 0.0;
            for (int e = tid; e < C::NR1; e += G)
            {
                int t, u, v;
                hermTuv(e, t, u, v);
                ht[e] = make_char4((char)t, (char)u, (char)v, (char)(t + u + v));
            }
            for (int e = tid; e < C::HAB; e += G)
            {
                int t, u, v;
                hermTuv(e, t, u, v);
                hab[e] = make_char4((char)t, (char)u, (char)v, 0);
            }
            for (int e = tid; e < C::HCD; e += G)
            {
                int t, u, v;
                hermTuv(e, t, u, v);
                hcd[e] = make_char4((char)t, (char)u, (char)v, (char)((t + u + v) & 1));
            }
        }
        __syncthreads();

        // E (x4 = 0) or E1_x (x4 = 1..3) of bra primitive p into a staged E_ab buffer, by cp.async
        auto issueE = [&](uint32_t p, int x4, double *dst) {
            const double *src = x4 == 0 ? a.bra.E + (size_t)p * C::SAB * C::HAB
                                        : a.bra.E1 + ((size_t)p * 3 + (x4 - 1)) * C::SAB * C::HAB;
            for (int e = tid; e < C::SAB * C::HAB; e += G)
                cpAsync8(dst + (e / C::HAB) * S::P_EA + e % C::HAB, src + e);
        };

        auto processTask = [&](uint32_t ib, uint32_t ik) {
            const int32_t *bi = a.bra.info + 8 * ib;
            const int32_t *ki = a.ket.info + 8 * ik;
            const uint32_t p0 = a.bra.pofs[ib], p1 = a.bra.pofs[ib + 1];
            // the first E matrix lands while Gamma is formed (the first buffer was last read by a
            // product that every thread finished before a later barrier)
            if constexpr (S::DB)
                issueE(p0, 0, ea);
            // Gamma[m][c] of the quartet (as in the block kernel's epilogues)
            {
                const int n = a.nao;
                const double *D = a.D;
                double w = 0.0;
                if (a.mode == kD1GradRI)
                {
                    const int32_t *mi = a.aux_side == 0 ? bi : ki;
                    w = a.aux_side == 2 ? -((a.same_class && ib == ik) ? 0.5 : 1.0) : (mi[4] == mi[5] ? 1.0 : 2.0);
                }
                else
                    w = quartetWeight(a, ib, ik);
                for (int e = tid; e < C::SAB * C::SCD; e += G)
                {
                    const int m = e / C::SCD, c = e % C::SCD;
                    double v;
                    if (a.mode == kD1GradRI)
                    {
                        if (a.aux_side == 2)
                            v = __ldg(a.dcoef + bi[0] + m) * __ldg(a.dcoef + ki[0] + c);
                        else if (a.aux_side == 0)
                            v = __ldg(D + (size_t)(bi[0] + m / C::SB) * n + bi[1] + m % C::SB) * __ldg(a.dcoef + ki[0] + c);
                        else
                            v = __ldg(D + (size_t)(ki[0] + c / C::SD) * n + ki[1] + c % C::SD) * __ldg(a.dcoef + bi[0] + m);
                    }
                    else
                    {
                        const size_t mu = bi[0] + m / C::SB, nu = bi[1] + m % C::SB;
                        const size_t ka = ki[0] + c / C::SD, ta = ki[1] + c % C::SD;
                        v = 4.0 * __ldg(D + mu * n + nu) * __ldg(D + ka * n + ta) - __ldg(D + mu * n + ka) * __ldg(D + nu * n + ta) -
                            __ldg(D + mu * n + ta) * __ldg(D + nu * n + ka);
                    }
                    gs[m * S::P_G + c] = w * v;
                }
            }
            double g[9];
#pragma unroll
            for (int x = 0; x < 9; x++)
                g[x] = 0.0;
            const uint32_t q0 = a.ket.pofs[ik], q1 = a.ket.pofs[ik + 1];
            for (uint32_t p = p0; p < p1; p++)
            {
                const PQ4 P = loadPQ(a.bra.pP, p);
                const double2 AB = __ldg(reinterpret_cast<const double2 *>(a.bra.ab) + p);
                // the first buffer's last reader (the x4 = 2 product of the previous primitive)
                // finished before the barriers of the ket loop
                if constexpr (S::DB)
                    if (p != p0)
                        issueE(p, 0, ea);
                // GE (x4 = 0) and GE1_x (x4 = 1..3) = E^T Gamma: with two buffers the next E matrix
                // lands during this product, else one staged E matrix at a time
                for (int x4 = 0; x4 < 4; x4++)
                {
                    const double *eb = ea;
                    if constexpr (S::DB)
                    {
                        cpAsyncWaitAll();  // E of this x4 (the only copy in flight)
                        __syncthreads();   // it is visible, Gamma is written, the product x4 - 1 is done
                        if (x4 < 3)
                            issueE(p, x4 + 1, (x4 & 1) ? ea : ea2);
                        eb = (x4 & 1) ? ea2 : ea;
                    }
                    else
                    {
                        const double *src = x4 == 0 ? a.bra.E + (size_t)p * C::SAB * C::HAB
                                                    : a.bra.E1 + ((size_t)p * 3 + (x4 - 1)) * C::SAB * C::HAB;
                        __syncthreads();  // the previous product has read ea (and, first time, gs is written)
                        for (int e = tid; e < C::SAB * C::HAB; e += G)
                            ea[(e / C::HAB) * S::P_EA + e % C::HAB] = __ldg(src + e);
                        __syncthreads();
                    }
                    double *out = ge + x4 * GE_SZ;
                    for (int t = warp; t < S::TILES1; t += WD)
                    {
                        const int mt = t / S::NT1, nt = t % S::NT1;
                        double d0 = 0.0, d1 = 0.0;
                        const double *A = eb + k4 * S::P_EA + mt * 8 + r8;
                        const double *B = gs + k4 * S::P_G + nt * 8 + r8;
#pragma unroll 4
                        for (int ks = 0; ks < S::KT1; ks++)
                            dmma8x8x4(d0, d1, A[ks * 4 * S::P_EA], B[ks * 4 * S::P_G]);
                        double *o = out + (mt * 8 + r8) * S::P_GE + nt * 8 + 2 * k4;
                        o[0] = d0;
                        o[1] = d1;
                    }
                }
                double t1[3] = {0, 0, 0}, t13[3] = {0, 0, 0}, tc[3] = {0, 0, 0};
                for (uint32_t q = q0; q < q1; q++)
                {
                    const PQ4 Q = loadPQ(a.ket.pP, q);
                    const double cq = __ldg(a.ket.ab + 2 * q) / Q.x;
                    const double rs = rsqrt(P.x + Q.x);
                    const double alpha = P.x * Q.x * (rs * rs);
                    const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                    const double fac = 34.986836655249725 * rs * P.ip * Q.ip;
                    double F[L1 + 1];
                    boysF<L1, false>(alpha * (X * X + Y * Y + Z * Z), a.boys + L1 * kBoysTerms * kBoysPitch, F);
                    const double m2a = -2.0 * alpha;
                    __syncthreads();  // the previous primitive's R and E tiles are no longer read
                    // ket E and E1 tiles [h'][c]
                    {
                        const double *ecd = a.ket.Et + (size_t)q * C::HCD * C::SCD;
                        const double *e1cd = a.ket.E1t + (size_t)q * 3 * C::HCD * C::SCD;
                        // copies land during the R build; waited for before the W products
                        for (int e = tid; e < C::HCD * C::SCD; e += G)
                        {
                            const int o = (e / C::SCD) * S::P_EC + e % C::SCD;
                            cpAsync8(ec + o, ecd + e);
                            cpAsync8(ec + EC_SZ + o, e1cd + e);
                            cpAsync8(ec + 2 * EC_SZ + o, e1cd + C::HCD * C::SCD + e);
                            cpAsync8(ec + 3 * EC_SZ + o, e1cd + 2 * C::HCD * C::SCD + e);
                        }
                    }
                    // R to order L + 1 (closed form, or levels split over the block)
                    double *cur = rb, *nxt = rb + C::NR1;
                    if constexpr (closedFormR<L1>())
                    {
                        groupHermiteR<L1, double>(F, fac, m2a, X, Y, Z, nxt, cur, ht, tid, G);
                    }
                    else
                    {
                    if (tid == 0)
                    {
                        double pw = 1.0;
                        for (int k = 0; k < L1; k++)
                            pw *= m2a;
                        cur[0] = F[L1] * fac * pw;
                    }
                    __syncthreads();
#pragma unroll
                    for (int nl = L1 - 1; nl >= 0; nl--)
                    {
                        const int cnt = nherm(L1 - nl);
                        for (int e = tid; e < cnt; e += G)
                        {
                            double r;
                            if (e == 0)
                            {
                                double pn = 1.0;
                                for (int k = 0; k < nl; k++)
                                    pn *= m2a;
                                r = F[nl] * fac * pn;
                            }
                            else
                            {
                                const char4 tv = ht[e];
                                const int t = tv.x, u = tv.y, v = tv.z, m = tv.w;
                                if (t > 0)
                                {
                                    r = X * cur[nherm(m - 2) + cartIndex(u, v)];
                                    if (t > 1)
                                        r += (t - 1) * cur[nherm(m - 3) + cartIndex(u, v)];
                                }
                                else if (u > 0)
                                {
                                    r = Y * cur[nherm(m - 2) + cartIndex(u - 1, v)];
                                    if (u > 1)
                                        r += (u - 1) * cur[nherm(m - 3) + cartIndex(u - 2, v)];
                                }
                                else
                                {
                                    r = Z * cur[nherm(m - 2) + cartIndex(0, v - 1)];
                                    if (v > 1)
                                        r += (v - 1) * cur[nherm(m - 3) + cartIndex(0, v - 2)];
                                }
                            }
                            nxt[e] = r;
                        }
                        __syncthreads();
                        double *tmp = cur;
                        cur = nxt;
                        nxt = tmp;
                    }
                    }
                    cpAsyncWaitAll();
                    __syncthreads();  // the ket tiles are visible to every warp
                    // the seven W products per tile, consumed in registers
                    double ax = 0, ay = 0, az = 0, c2x = 0, c2y = 0, c2z = 0;
                    for (int t = warp; t < S::TILES2; t += WD)
                    {
                        const int mt = t / S::NT2, nt = t % S::NT2;
                        double w[7][2];
#pragma unroll
                        for (int k = 0; k < 7; k++)
                            w[k][0] = w[k][1] = 0.0;
                        const double *A = ge + (mt * 8 + r8) * S::P_GE + k4;
                        const double *B = ec + (nt * 8 + r8) * S::P_EC + k4;
#pragma unroll 2
                        for (int ks = 0; ks < S::KT2; ks++)
                        {
                            const double a0 = A[ks * 4], a1 = A[GE_SZ + ks * 4], a2 = A[2 * GE_SZ + ks * 4],
                                         a3 = A[3 * GE_SZ + ks * 4];
                            const double b0 = B[ks * 4], b1 = B[EC_SZ + ks * 4], b2 = B[2 * EC_SZ + ks * 4],
                                         b3 = B[3 * EC_SZ + ks * 4];
                            dmma8x8x4(w[0][0], w[0][1], a0, b0);
                            dmma8x8x4(w[1][0], w[1][1], a1, b0);
                            dmma8x8x4(w[2][0], w[2][1], a2, b0);
                            dmma8x8x4(w[3][0], w[3][1], a3, b0);
                            dmma8x8x4(w[4][0], w[4][1], a0, b1);
                            dmma8x8x4(w[5][0], w[5][1], a0, b2);
                            dmma8x8x4(w[6][0], w[6][1], a0, b3);
                        }
                        const int h = mt * 8 + r8;
                        if (h < C::HAB)
                        {
                            const char4 th = hab[h];
#pragma unroll
                            for (int j = 0; j < 2; j++)
                            {
                                const int hp = nt * 8 + 2 * k4 + j;
                                if (hp < C::HCD)
                                {
                                    const char4 tp = hcd[hp];
                                    const int tt = th.x + tp.x, uu = th.y + tp.y, vv = th.z + tp.z;
                                    const double sg = tp.w ? -1.0 : 1.0;
                                    const double r0 = sg * cur[hermIndex(tt, uu, vv)];
                                    const double rx = sg * cur[hermIndex(tt + 1, uu, vv)];
                                    const double ry = sg * cur[hermIndex(tt, uu + 1, vv)];
                                    const double rz = sg * cur[hermIndex(tt, uu, vv + 1)];
                                    ax += w[0][j] * rx;
                                    ay += w[0][j] * ry;
                                    az += w[0][j] * rz;
                                    t13[0] += w[1][j] * r0;
                                    t13[1] += w[2][j] * r0;
                                    t13[2] += w[3][j] * r0;
                                    c2x += w[4][j] * r0;
                                    c2y += w[5][j] * r0;
                                    c2z += w[6][j] * r0;
                                }
                            }
                        }
                    }
                    t1[0] += ax;
                    t1[1] += ay;
                    t1[2] += az;
                    tc[0] += c2x - cq * ax;
                    tc[1] += c2y - cq * ay;
                    tc[2] += c2z - cq * az;
                }
                const double ap = AB.x * P.ip, bp = AB.y * P.ip;
#pragma unroll
                for (int x = 0; x < 3; x++)
                {
                    g[x] += ap * t1[x] + t13[x];
                    g[3 + x] += bp * t1[x] - t13[x];
                    g[6 + x] += tc[x];
                }
            }
            // the 9 sums over the block, then per atom (D by translational invariance)
#pragma unroll
            for (int x = 0; x < 9; x++)
            {
                double v = g[x];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0)
                    red[warp * 9 + x] = v;
            }
            __syncthreads();
            if (tid < 9)
            {
                double v = 0.0;
                for (int w = 0; w < WD; w++)
                    v += red[w * 9 + tid];
                const int centre = tid / 3, x = tid % 3;
                const int atom = centre == 0 ? bi[2] : centre == 1 ? bi[3] : ki[2];
                atomicAdd(a.grad + 3 * atom + x, v);
                atomicAdd(a.grad + 3 * ki[3] + x, -v);
            }
            __syncthreads();
        };

        // the block's tasks come in increasing order, so one forward-moving cursor decodes them
        int cur = 0;
        auto runTask = [&](long long task) {
            uint32_t ib, ik;
            decodeCursor(a, task, cur, ib, ik);
            if (inWindow(a, ib, ik, 0, false))
                processTask(ib, ik);
        };
        if (a.chunks)
        {
            __shared__ unsigned long long claimed;
            for (;;)
            {
                if (tid == 0)
                    claimed = atomicAdd(a.counter, 1ULL);
                __syncthreads();
                const unsigned long long c = claimed;
                __syncthreads();
                if (c >= (unsigned long long)a.n_chunks)
                    break;
                const long long t1 = (long long)__ldg(a.chunks + c + 1);
                for (long long t = (long long)__ldg(a.chunks + c); t < t1; t++)
                    runTask(t);
            }
        }
        else
            for (long long task = blockIdx.x; task < a.n_tasks; task += gridDim.x)
                runTask(task);
    }
}
