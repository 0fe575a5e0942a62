// batch_resident.cu -- the batched solver's cluster-resident kernel (K4r).
//
// The single-system SM-resident kernel (pcg_resident.cu, pcg_resident1_kernel) applied per
// system to the CTAs of one thread-block cluster.  A cluster pops a system from the device
// work queue and splits its slices into contiguous bands, one per CTA.  Each CTA keeps in
// shared memory, for the whole solve of that system: the window of the search direction p'
// that its band's columns reach (own band + halo), and r, Ap', the FP32 increment dx of x,
// M^-1 and the row sums of its own rows.  The SpMV gathers p' from shared memory; the global
// streams are the matrix and the halo's records.
//
// One cluster barrier per iteration.  As in pcg_resident1_kernel, the dot products of the
// next r.z and r.r are expanded in alpha, the seven partials reduced together (through
// distributed shared memory, in cluster-rank order, so every CTA takes the same decisions),
// and each row that another CTA's window covers publishes {M r, M Ap', p'} to double-buffered
// global records from which the reader rebuilds p'_new with the owner's fused multiply-adds,
// bit for bit.  Records cross SMs through L2 (loads with .cg, after the barrier's
// release/acquire at cluster scope).  Control flow, breakdown tests and status codes as the
// global-memory batch kernel (kernels/cuper_pcg_control_kernel.cpp:1069-1235).
//
// Dynamic shared memory per CTA (bytes): 16-aligned slice table (8 per slice) | p' window
// (4 wn) | r | Ap' | dx | M^-1 | row sums (4 nb each) | (when it fits the rest of the
// launch's budget) the band's own matrix: values, then columns, slot for slot as in global
// memory.  A CTA whose band's matrix is staged there reads no global memory in the SpMV; the
// products are the same, in the same order.  The host sizes each launch for the largest band
// among the systems it routes there (and widens it to the most that keeps the launch's
// occupancy, so that matrices fit); a system that would not fit is skipped with
// iterations = -1, which the host reports as an error.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "batch_common.cuh"
#include "device_common.cuh"
#include "pcg_device.cuh"

namespace xplus {
namespace {

using namespace dev;

constexpr int kBrPartials = 7;

template <typename VT, int CHUNK, typename IT>
__global__ void __launch_bounds__(512, 1) pcg_batch_res_kernel(BatchArgs a) {
    constexpr int NS = 4;  // slices of one warp in flight together in the SpMV
    // halo float4 groups per thread loaded ahead (per record array): as many as fit 128
    // registers without spills (-Xptxas -v)
    constexpr int kHaloU = std::is_same<VT, float>::value ? 3 : 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_red[32 * kBrPartials];
    __shared__ double s_part[2][8];
    __shared__ double s_tot[8];
    __shared__ int s_item[2];
    __shared__ int s_mm[2][32];
    __shared__ int s_win[4];   // this CTA's w0, wn, fits, matrix staged (read by the other CTAs)
    __shared__ int s_sys[4];   // exp_lo, exp_hi, every CTA fits, CTAs that staged their matrix
    cg::cluster_group cl = cg::this_cluster();
    const int crank = static_cast<int>(cl.block_rank());
    const int csize = static_cast<int>(cl.num_blocks());
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const IT* __restrict__ col = static_cast<const IT*>(a.col);
    const size_t R = static_cast<size_t>(a.rows);
    int pbank = 0, ibank = 0;

    // cluster totals: block sums into this CTA's s_part[pbank] (publish), the cluster barrier,
    // then every CTA sums all ranks' partials in rank order (collect)
    auto publish = [&](const auto& v) {
        constexpr int NV = static_cast<int>(std::extent<std::remove_reference_t<decltype(v)>>::value);
        block_sum_scatter<NV>(v, s_red, [&](int q, double x) { s_part[pbank][q] = x; });
    };
    auto collect = [&](int nv) {
        if (threadIdx.x < nv) {
            double t = 0.0;
            for (int rk = 0; rk < csize; ++rk) t += *cl.map_shared_rank(&s_part[pbank][threadIdx.x], rk);
            s_tot[threadIdx.x] = t;
        }
        __syncthreads();
        pbank ^= 1;
    };

    for (;;) {
        if (crank == 0 && threadIdx.x == 0) s_item[ibank] = a.q_begin + atomicAdd(a.head, 1);
        cl.sync();
        const int qi = *cl.map_shared_rank(&s_item[ibank], 0);
        ibank ^= 1;
        if (qi >= a.q_end) {
            // every CTA has read rank 0's queue item before any CTA of the cluster exits: a
            // CTA's shared memory must outlive all distributed-shared-memory reads of it
            cl.sync();
            break;
        }
        const long long t_begin = globaltimer_ns();
        const int sys = a.order[qi];
        const int S0 = a.sys_slice0[sys];
        const int ns = a.sys_slice0[sys + 1] - S0;
        const int per = (ns + csize - 1) / csize;
        const int sb = S0 + min(ns, crank * per);
        const int se = S0 + min(ns, (crank + 1) * per);
        const int nsl = se - sb;
        const int r0 = sb * 32;
        const int nb = nsl * 32;
        const int n = a.sys_n[sys];
        const float vscale = a.sys_scale[sys];
        const int max_iters = a.max_iters > 0 ? a.max_iters : max(4 * n, 1000);
        const bool true_mode = a.tau_mode == XPLUS_TAU_REL_TRUE;

        // ---- the band's window: the rows its columns reach, widened to float4 groups ----
        {
            int cmin = r0, cmax = r0 + nb;  // [cmin, cmax)
            for (int s = sb + warp; s < se; s += wpb) {
                const long long b0 = a.slice_ptr[s];
                const int w = static_cast<int>((a.slice_ptr[s + 1] - b0) >> 5);
                const int row = s * 32 + lane;
                for (int c = 0; c < w; c += CHUNK) {
                    int cc[CHUNK];
                    ColLoad<CHUNK, IT>::run(col + b0 + static_cast<long long>(c) * 32 + lane * CHUNK, row, cc);
#pragma unroll
                    for (int q = 0; q < CHUNK; ++q) {
                        cmin = min(cmin, cc[q]);
                        cmax = max(cmax, cc[q] + 1);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
                cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
            }
            if (lane == 0) {
                s_mm[0][warp] = cmin;
                s_mm[1][warp] = cmax;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int w = 1; w < wpb; ++w) {
                    cmin = min(cmin, s_mm[0][w]);
                    cmax = max(cmax, s_mm[1][w]);
                }
                const int w0 = max(S0 * 32, cmin & ~3);
                const int wend = min((S0 + ns) * 32, (cmax + 3) & ~3);
                const long long need = ((static_cast<long long>(nsl) * 8 + 15) & ~15LL) +
                                       4LL * (static_cast<long long>(wend - w0) + 5LL * nb);
                // the band's slots (a multiple of 32 per slice, so both arrays are whole
                // 16-byte groups)
                const long long ms = a.slice_ptr[se] - a.slice_ptr[sb];
                const long long mat = ms * static_cast<long long>(sizeof(VT) + sizeof(IT));
                s_win[0] = w0;
                s_win[1] = wend - w0;
                s_win[2] = need <= a.res_smem ? 1 : 0;
                s_win[3] = a.stage_matrix && need + mat <= a.res_smem ? 1 : 0;
            }
        }
        // every CTA's window: the rows of this band that others read, and whether all fit
        cl.sync();
        if (threadIdx.x == 0) {
            int lo = r0, hi = r0 + nb, fit = 1, staged = 0;
            for (int rk = 0; rk < csize; ++rk) {
                const int* wk = cl.map_shared_rank(s_win, rk);
                const int wx = wk[0], wy = wk[1];
                fit &= wk[2];
                staged += wk[3];
                if (rk == crank || wy <= 0) continue;
                if (rk < crank) lo = max(lo, wx + wy);
                else hi = min(hi, wx);
            }
            s_sys[0] = min(lo, r0 + nb);
            s_sys[1] = max(hi, r0);
            s_sys[2] = fit;
            s_sys[3] = staged;
        }
        __syncthreads();
        if (!s_sys[2]) {
            // the host sizes each launch for every system it routes there, so this is not
            // reached; skipped rather than overrun shared memory, and reported (iterations -1)
            if (crank == 0 && threadIdx.x == 0) {
                a.out_status[sys] = XPLUS_BREAKDOWN;
                a.out_iters[sys] = -1;
                a.out_repl[sys] = 0;
                a.out_true_rel[sys] = -1.0;
                a.out_ns[sys] = 0;
                if (a.out_staged) a.out_staged[sys] = 0;
            }
            continue;
        }
        const int w0 = s_win[0], wn = s_win[1];
        const bool staged = s_win[3] != 0;
        const int exp_lo = s_sys[0], exp_hi = s_sys[1];
        int2* s_slice = reinterpret_cast<int2*>(smem_raw);
        float* pw = reinterpret_cast<float*>(smem_raw + ((static_cast<size_t>(nsl) * 8 + 15) & ~static_cast<size_t>(15)));
        float* rv = pw + wn;
        float* apv = rv + nb;
        float* dxv = apv + nb;
        float* mi = dxv + nb;
        float* rsv = mi + nb;
        // the staged matrix (16-aligned: the vectors end on a 16-byte boundary, wn being a
        // multiple of 4 and nb of 32); slice offsets then count from the band's first slot
        const long long m0 = a.slice_ptr[sb];
        const long long ms = a.slice_ptr[se] - m0;
        VT* mval = reinterpret_cast<VT*>(rsv + nb);
        IT* mcol = reinterpret_cast<IT*>(mval + ms);
        for (int k = threadIdx.x; k < nsl; k += blockDim.x) {
            const long long b0 = a.slice_ptr[sb + k];
            s_slice[k] = make_int2(static_cast<int>(staged ? b0 - m0 : b0),
                                   static_cast<int>((a.slice_ptr[sb + k + 1] - b0) >> 5));
        }
        if (staged) {
            const uint4* gv = reinterpret_cast<const uint4*>(val + m0);
            const uint4* gc = reinterpret_cast<const uint4*>(col + m0);
            uint4* sv = reinterpret_cast<uint4*>(mval);
            uint4* sc = reinterpret_cast<uint4*>(mcol);
            const long long nv = ms * static_cast<long long>(sizeof(VT)) / 16;
            const long long nc = ms * static_cast<long long>(sizeof(IT)) / 16;
            for (long long i = threadIdx.x; i < nv; i += blockDim.x) sv[i] = __ldg(gv + i);
            for (long long i = threadIdx.x; i < nc; i += blockDim.x) sc[i] = __ldg(gc + i);
        }
        for (int t = threadIdx.x; t < nb; t += blockDim.x) {
            mi[t] = a.minv[r0 + t];
            rsv[t] = a.rowsum[r0 + t];
            dxv[t] = 0.0f;
            apv[t] = 0.0f;
        }
        for (int t = threadIdx.x; t < wn; t += blockDim.x) pw[t] = 0.0f;
        __syncthreads();
        auto rec_zr = [&](int g) { return a.rec3 + (3 * static_cast<size_t>(g) + 0) * R; };
        auto rec_za = [&](int g) { return a.rec3 + (3 * static_cast<size_t>(g) + 1) * R; };
        auto rec_p = [&](int g) { return a.rec3 + (3 * static_cast<size_t>(g) + 2) * R; };
        auto flush_dx = [&]() {
            for (int t = threadIdx.x; t < nb; t += blockDim.x) {
                a.x64[r0 + t] += static_cast<double>(dxv[t]);
                dxv[t] = 0.0f;
            }
        };
        // r = b - A x in FP64 (x of neighbours through L2) into shared r; records of
        // generation g get {m r, 0, p (kept, or 0 when init)}; sums r.z, r.r, ||b - A x||^2,
        // ||b||^2 (init)
        auto residual_phase = [&](bool init, int g) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int s = sb + warp; s < se; s += wpb) {
                const int row = s * 32 + lane;
                const double bv = a.b64[row];
                const double rt = bv - batch_row64<CHUNK, IT>(a, s, lane);
                const float r_ = static_cast<float>(rt);
                const float z_ = mi[row - r0] * r_;
                if (init) acc[3] += bv * bv;
                rv[row - r0] = r_;
                rec_zr(g)[row] = z_;
                rec_za(g)[row] = 0.0f;
                if (init) rec_p(g)[row] = 0.0f;
                acc[0] += static_cast<double>(r_) * static_cast<double>(z_);
                acc[1] += static_cast<double>(r_) * static_cast<double>(r_);
                acc[2] += rt * rt;
            }
            publish(acc);
            cl.sync();
            collect(4);
        };
        auto apply_update = [&](float al) {
            for (int t = threadIdx.x; t < nb; t += blockDim.x) {
                const float pv = pw[r0 + t - w0];
                dxv[t] = __fmaf_rn(al, pv, dxv[t]);
                rv[t] = rv[t] - al * apv[t];
            }
        };
        // the halo's records in float4 groups (group u < nlo below the band, the rest above)
        const int nlo = (r0 - w0) >> 2;
        const int hi0 = (r0 + nb - w0) >> 2;
        const int nh = nlo + (wn >> 2) - hi0;
        const int hbd = static_cast<int>(blockDim.x);
        auto qof = [&](int u) { return u < nlo ? u : hi0 + (u - nlo); };
        float4 hz[kHaloU], hq[kHaloU], hp[kHaloU];
        auto issue_halo = [&](int g) {
            const float4* zr4 = reinterpret_cast<const float4*>(rec_zr(g) + w0);
            const float4* za4 = reinterpret_cast<const float4*>(rec_za(g) + w0);
            const float4* p4 = reinterpret_cast<const float4*>(rec_p(g) + w0);
#pragma unroll
            for (int v = 0; v < kHaloU; ++v) {
                const int u = threadIdx.x + v * hbd;
                if (u < nh) {
                    const int qq = qof(u);
                    hz[v] = __ldcg(zr4 + qq);
                    hq[v] = __ldcg(za4 + qq);
                    hp[v] = __ldcg(p4 + qq);
                }
            }
        };
        bool halo_ready = false;

        int gen = 0;
        residual_phase(true, gen);
        issue_halo(gen);
        halo_ready = true;
        double rz = s_tot[0], rr = s_tot[1], true_rr = s_tot[2];
        const double bb = s_tot[3];
        const double tau_true_rr = a.tau * a.tau * bb;
        double rr_at_replace = rr;
        double pap = 0.0, alpha = 0.0, beta = 0.0;
        double pend = 0.0;  // alpha of the update not yet applied to x and r (0: none)
        int status = XPLUS_MAX_ITER, iterations = 0, replacements = 0;
        bool stagnated = false;
        ReplacePolicy pol(a.restart_on_replace, true_rr);
        const bool converged_now = true_mode ? (true_rr <= tau_true_rr) : (rr <= a.tau);
        constexpr int kFlushEvery = 16;

        if (converged_now) {
            status = XPLUS_CONVERGED;
        } else {
            for (int it = 0; it < max_iters; ++it) {
                if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                    status = XPLUS_BREAKDOWN;
                    break;
                }
                // ---- the previous update and the new p': own band from shared memory (the
                // records this CTA published hold these very values), halo from the records ----
                if (!halo_ready) issue_halo(gen);
                halo_ready = false;
                const float al_prev = static_cast<float>(pend);
                const bool upd = pend != 0.0;
                const bool flush = upd && it % kFlushEvery == 0;
                const float be = static_cast<float>(beta);
                {
                    // four rows per thread and step (float4: pw + r0 - w0 and the band's arrays
                    // start on 16-byte boundaries, w0 being a multiple of 4 and nb of 32); each
                    // row's arithmetic is the scalar form's
                    float4* pw4o = reinterpret_cast<float4*>(pw + (r0 - w0));
                    float4* rv4 = reinterpret_cast<float4*>(rv);
                    const float4* ap4 = reinterpret_cast<const float4*>(apv);
                    const float4* mi4 = reinterpret_cast<const float4*>(mi);
                    float4* dx4 = reinterpret_cast<float4*>(dxv);
                    auto row_update = [&](float& pv, float& r_, float ap_, float m, float& d) {
                        const float mr = m * r_;
                        const float ma = upd ? m * ap_ : 0.0f;  // the records' m Ap' is 0 after a residual
                        const float pn = __fmaf_rn(be, pv, __fmaf_rn(-al_prev, ma, mr));
                        if (upd) {
                            d = __fmaf_rn(al_prev, pv, d);
                            r_ = r_ - al_prev * ap_;
                        }
                        pv = pn;
                    };
                    for (int t4 = threadIdx.x; t4 < (nb >> 2); t4 += blockDim.x) {
                        float4 pv = pw4o[t4];
                        float4 r4 = rv4[t4];
                        const float4 a4 = ap4[t4], m4 = mi4[t4];
                        float4 d4 = upd ? dx4[t4] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        row_update(pv.x, r4.x, a4.x, m4.x, d4.x);
                        row_update(pv.y, r4.y, a4.y, m4.y, d4.y);
                        row_update(pv.z, r4.z, a4.z, m4.z, d4.z);
                        row_update(pv.w, r4.w, a4.w, m4.w, d4.w);
                        pw4o[t4] = pv;
                        if (upd) {
                            rv4[t4] = r4;
                            if (flush) {
                                double* xr = a.x64 + r0 + 4 * t4;
                                xr[0] += static_cast<double>(d4.x);
                                xr[1] += static_cast<double>(d4.y);
                                xr[2] += static_cast<double>(d4.z);
                                xr[3] += static_cast<double>(d4.w);
                                d4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                            }
                            dx4[t4] = d4;
                        }
                    }
                }
                pend = 0.0;
                {
                    const float4* zr4 = reinterpret_cast<const float4*>(rec_zr(gen) + w0);
                    const float4* za4 = reinterpret_cast<const float4*>(rec_za(gen) + w0);
                    const float4* p4 = reinterpret_cast<const float4*>(rec_p(gen) + w0);
                    float4* pw4 = reinterpret_cast<float4*>(pw);
                    auto fill = [&](const float4& z, const float4& q, const float4& p) {
                        float4 o;
                        o.x = __fmaf_rn(be, p.x, __fmaf_rn(-al_prev, q.x, z.x));
                        o.y = __fmaf_rn(be, p.y, __fmaf_rn(-al_prev, q.y, z.y));
                        o.z = __fmaf_rn(be, p.z, __fmaf_rn(-al_prev, q.z, z.z));
                        o.w = __fmaf_rn(be, p.w, __fmaf_rn(-al_prev, q.w, z.w));
                        return o;
                    };
#pragma unroll
                    for (int v = 0; v < kHaloU; ++v) {
                        const int u = threadIdx.x + v * hbd;
                        if (u < nh) pw4[qof(u)] = fill(hz[v], hq[v], hp[v]);
                    }
                    for (int u = threadIdx.x + kHaloU * hbd; u < nh; u += hbd) {
                        const int qq = qof(u);
                        pw4[qq] = fill(__ldcg(zr4 + qq), __ldcg(za4 + qq), __ldcg(p4 + qq));
                    }
                    __syncthreads();
                }
                // ---- Ap' from shared memory, each row's records of the next generation (rows
                // that other CTAs read) and its terms of the seven sums ----
                {
                    double acc[kBrPartials] = {0, 0, 0, 0, 0, 0, 0};
                    const int g1 = gen ^ 1;
                    float* zr1 = rec_zr(g1);
                    float* za1 = rec_za(g1);
                    float* p1 = rec_p(g1);
                    for (int s0 = sb + warp; s0 < se; s0 += NS * wpb) {
                        int2 sl[NS];
                        int row[NS];
                        float pi[NS], y[NS];
#pragma unroll
                        for (int k = 0; k < NS; ++k) {
                            const int s = s0 + k * wpb;
                            const bool on = s < se;
                            sl[k] = on ? s_slice[s - sb] : make_int2(0, 0);
                            row[k] = on ? s * 32 + lane : -1;
                            pi[k] = on ? pw[row[k] - w0] : 0.0f;
                        }
                        // one generic load path for both homes of the matrix
                        sell_rows_smem<VT, CHUNK, IT, NS, kLdPlain>(sl, row, lane, staged ? mcol : col,
                                                                    staged ? mval : val, pw, w0, pi, y);
#pragma unroll
                        for (int k = 0; k < NS; ++k) {
                            if (row[k] < 0) continue;
                            const int t = row[k] - r0;
                            const float ap_ = y[k] * vscale + rsv[t] * pi[k];
                            apv[t] = ap_;
                            const float r_ = rv[t], m = mi[t];
                            if (row[k] < exp_lo || row[k] >= exp_hi) {
                                zr1[row[k]] = m * r_;
                                za1[row[k]] = m * ap_;
                                p1[row[k]] = pi[k];
                            }
                            const double dr = r_, da = ap_, dm = m;
                            acc[0] += static_cast<double>(pi[k]) * da;
                            acc[1] += dm * dr * dr;
                            acc[2] += dm * dr * da;
                            acc[3] += dm * da * da;
                            acc[4] += dr * dr;
                            acc[5] += dr * da;
                            acc[6] += da * da;
                        }
                    }
                    publish(acc);
                }
                cl.sync();
                issue_halo(gen ^ 1);  // the generation just published
                halo_ready = true;
                collect(kBrPartials);
                gen ^= 1;
                pap = s_tot[0];
                if (bad(pap) || fabs(pap) <= kBreakdownEps) {
                    status = XPLUS_BREAKDOWN;
                    break;
                }
                const double rz_old = rz;
                alpha = rz / pap;
                if (bad(alpha)) {
                    status = XPLUS_BREAKDOWN;
                    break;
                }
                pend = alpha;
                double rz_new = s_tot[1] - 2.0 * alpha * s_tot[2] + alpha * alpha * s_tot[3];
                double rr_new = s_tot[4] - 2.0 * alpha * s_tot[5] + alpha * alpha * s_tot[6];
                iterations = it + 1;
                if (bad(rz_new) || bad(rr_new)) {
                    rz = rz_new;
                    rr = rr_new;
                    status = XPLUS_BREAKDOWN;
                    break;
                }
                bool do_replace = false, drop_replace = false;
                double zap = 0.0;  // z_new . Ap' of a replacement
                if (true_mode) {
                    if (rr_new <= tau_true_rr) do_replace = drop_replace = true;
                    if (a.replace_every > 0 && iterations % a.replace_every == 0) do_replace = true;
                    if (a.replace_drop2 > 0.0 && rr_new <= a.replace_drop2 * rr_at_replace) do_replace = drop_replace = true;
                }
                if (do_replace) {
                    halo_ready = false;  // the residual phase rewrites this generation's records
                    apply_update(static_cast<float>(pend));
                    pend = 0.0;
                    __syncthreads();
                    flush_dx();
                    cl.sync();
                    residual_phase(false, gen);
                    rz_new = s_tot[0];
                    rr_new = s_tot[1];
                    true_rr = s_tot[2];
                    ++replacements;
                    rr_at_replace = rr_new;
                    if (pol.after(a.restart_on_replace, true_rr, a.stag_factor, a.stag_window)) stagnated = true;
                    if (pol.mode == 4) {
                        // z_new . Ap' for the flexible coefficient (each thread reads back only
                        // the records it wrote)
                        double acc[1] = {0.0};
                        for (int s = sb + warp; s < se; s += wpb) {
                            const int row = s * 32 + lane;
                            acc[0] += static_cast<double>(rec_zr(gen)[row]) * static_cast<double>(apv[row - r0]);
                        }
                        publish(acc);
                        cl.sync();
                        collect(1);
                        zap = s_tot[0];
                    }
                }
                rz = rz_new;
                rr = rr_new;
                if (true_mode ? (do_replace && true_rr <= tau_true_rr) : (rr <= a.tau)) {
                    status = XPLUS_CONVERGED;
                    break;
                }
                if (stagnated) break;
                if (fabs(rz_old) <= kBreakdownEps) {
                    status = XPLUS_BREAKDOWN;
                    break;
                }
                beta = pol.beta(do_replace, drop_replace, rz, rz_old, zap, pap);
                if (bad(beta)) {
                    status = XPLUS_BREAKDOWN;
                    break;
                }
            }
        }
        if (status == XPLUS_MAX_ITER && !true_mode && rr <= a.tau) status = XPLUS_CONVERGED;

        // ---- exit: the pending update, dx into x, then the FP64 true residual ----
        if (pend != 0.0) {
            apply_update(static_cast<float>(pend));
            __syncthreads();
        }
        flush_dx();
        cl.sync();
        {
            double fin[1] = {0.0};
            for (int s = sb + warp; s < se; s += wpb) {
                const int row = s * 32 + lane;
                const double rt = a.b64[row] - batch_row64<CHUNK, IT>(a, s, lane);
                fin[0] += rt * rt;
            }
            publish(fin);
            cl.sync();
            collect(1);
        }
        if (crank == 0 && threadIdx.x == 0) {
            a.out_status[sys] = status;
            a.out_iters[sys] = iterations;
            a.out_repl[sys] = replacements;
            a.out_true_rel[sys] = bb > 0.0 ? sqrt(s_tot[0] / bb) : sqrt(s_tot[0]);
            a.out_ns[sys] = globaltimer_ns() - t_begin;
            if (a.out_staged) a.out_staged[sys] = s_sys[3];
        }
    }
}

template <typename VT, typename IT>
BatchKernel pick_res_chunk(int chunk) {
    switch (chunk) {
        case 1: return pcg_batch_res_kernel<VT, 1, IT>;
        case 2: return pcg_batch_res_kernel<VT, 2, IT>;
        case 4: return pcg_batch_res_kernel<VT, 4, IT>;
    }
    return nullptr;
}

template <typename IT>
BatchKernel pick_res_vt(int vt, int chunk) {
    switch (vt) {
        case XPLUS_F32: return pick_res_chunk<float, IT>(chunk);
        case XPLUS_BF16: return pick_res_chunk<__nv_bfloat16, IT>(chunk);
        case XPLUS_F16: return pick_res_chunk<__half, IT>(chunk);
    }
    return nullptr;
}

}  // namespace

BatchKernel batch_resident_kernel(int vt, int chunk, bool idx16) {
    return idx16 ? pick_res_vt<short>(vt, chunk) : pick_res_vt<int>(vt, chunk);
}

int batch_resident_static_smem(BatchKernel k) {
    cudaFuncAttributes fa{};
    if (!k || cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(k)) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return static_cast<int>(fa.sharedSizeBytes);
}

}  // namespace xplus
