// translate_tiled.cu -- the pair translation pass for clusters whose spheres
// all have one order L (the fast path; mixed orders use translate.cu).
//
// Same mathematics as translate.cu (MSTM's coefficient_translation,
// december2023/mstm-modules-33.f90:6610-6787, applied in both directions per
// pair as in external_to_external_expansion, modules:6390-6525), organised for
// throughput:
//   * L and the number of right-hand sides NR are template parameters, so every
//     index is a compile-time expression and every short loop unrolls;
//   * pairs are grouped in tiles: all pairs (i, j) with i in sphere block I
//     and j in block J (B spheres per block).  A CTA works through whole tiles
//     and accumulates the outputs of the tile's 2B spheres in shared memory,
//     flushing them to y with coalesced vector atomics once per tile;
//   * per pair the work is four small dense products over C = 4*NR columns
//     (direction x rhs x mode), each output computed from a matrix row or
//     column held in registers:
//        A  shift/phase/even-odd split of the sources          (C x L(L+3)/2)
//        B  forward rotation  [P;Q] = [E;O] [S;T]               per degree n
//        C  axial translation  g = Z a'  (Z^T a' for i -> j)     per degree m
//        D  back rotation + phase + shift, accumulated in smem   per degree n
//   * the operator record of the next pair streams in with a bulk TMA copy
//     (cp.async.bulk + mbarrier) while the current one is applied;
//   * more than NR right-hand sides are split in chunks of NR columns; a work
//     item is (tile, chunk) with the chunk varying fastest, so the CTAs that
//     run the chunks of one tile at the same time read its operator records
//     from L2 after the first one brought them from HBM.
#include "common.cuh"
#include "kernels.cuh"
#include "translate_tiled.cuh"
#include "pairpipe.cuh"

using namespace pairpipe;

namespace {

// degree offsets in the packed per-column arrays
__host__ __device__ constexpr int sofs(int n) { return (n - 1) * (n + 2) / 2; }   // S/P: m = 0..n
__host__ __device__ constexpr int tofs(int n) { return (n - 1) * n / 2; }         // T/Q: m = 1..n

}  // namespace

// CTAs per SM the register budget is sized for: 3 for FP32 with one or two
// columns (80 registers; the extra resident warps hide the pass's latencies:
// fractal500 FP32, 2 columns, 2.27 -> 1.88 ms) and for FP64 up to order 7
// (FP64, 2 columns: 1500 spheres of order 5 16.5 -> 14.7 ms, 1000 of order 6
// 8.32 -> 7.62 ms, 800 of order 7 6.01 -> 5.58 ms), 2 otherwise
// (FP64 at larger orders and four FP32 columns slow down at the smaller
// budget: fractal500 FP64, 2 columns, 2.9 -> 4.1 ms).  FP64 below order 5
// runs the order-generic kernel, faster there than this one at either budget.
// With two pairs a step the shared memory holds two CTAs per SM, which get
// the 128-register budget.
// Column stride (complex values) of the sources, S/T, a', g and tile-output
// columns in shared memory: L(L+2), or for even L (a multiple of 8) one more
// (FP64: 16-byte values, 4 banks apart) or two more (FP32, 16-byte aligned)
// so that the columns a group of lanes reads at once fall on different banks
template <typename T> __host__ __device__ constexpr int tiled_cs(int L)
{
    return (L & 1) ? L * (L + 2) : L * (L + 2) + (sizeof(T) == 8 ? 1 : 2);
}

template <typename T, int L, int NR, int PP> __host__ __device__ constexpr int tiled_minb()
{
    return ((sizeof(T) == 4 && NR <= 2 && PP == 1) || (sizeof(T) == 8 && L <= 7)) ? 3 : 2;
}

// One CTA works through whole tiles, PP pairs of a tile at a time (a step):
// consecutive pairs whose output slots are disjoint share one step, so the
// four phases and their barriers serve both (PP = 2), which fills the
// threads of the rotation phases and halves the barriers per pair.
template <typename T, int L, int NR, int B, int PP, bool SO, int MB>
__global__ void __launch_bounds__(256, MB) translate_tiled_kernel(TiledArgs<T> a)
{
    constexpr int NT = 256;
    constexpr int C = 4 * NR;            // columns of a pair: ((dir*NR)+r)*2+p
    constexpr int CB = 4;                // columns per item in the rotations
    constexpr int NG = C / CB;
    constexpr int NS = L * (L + 3) / 2;  // (n, k>=0) rows
    constexpr int NQ = L * (L + 1) / 2;
    constexpr int NB2 = L * (L + 2);     // NS + NQ: one mode of a sphere block
    constexpr int NB = 2 * NB2;
    constexpr int REC = op_record_units(L, L);
    constexpr int RS = op_rot_size(L, L);
    constexpr int NSLOT = 2 * B;
    constexpr uint32_t RECB = (uint32_t)(REC * sizeof(T));
    constexpr uint32_t XB = (uint32_t)(NB * sizeof(cpx<T>));   // one sphere block of one rhs
    constexpr uint32_t XB2 = (uint32_t)(NB2 * sizeof(cpx<T>)); // one mode of it
    constexpr int CS = tiled_cs<T>(L);   // column stride of W1 / W2 / ACC (bank-spread for even L)
    constexpr int WP = C * CS;           // one pair's share of W1 / W2

    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);          // [0],[1] operators, [2] sources
    short2* tabS = reinterpret_cast<short2*>(sm + 64);        // NS entries (n, k), n descending
    short2* tabQ = tabS + NS;                                  // NQ entries (n, m>=1)
    short2* tabC = tabQ + NQ;                                  // NS entries (m, line), m = 0..L, line = max(1,m)..L
    size_t off = 64 + sizeof(short2) * (NS + NQ + NS);
    off = (off + 127) & ~(size_t)127;
    cpx<T>* ephm = reinterpret_cast<cpx<T>*>(sm + off);       // PP x (2L+1)
    off += sizeof(cpx<T>) * PP * (2 * L + 1);
    off = (off + 127) & ~(size_t)127;
    T* opb = reinterpret_cast<T*>(sm + off);                  // 2 buffers x PP records
    off += sizeof(T) * 2 * PP * REC;
    off = (off + 127) & ~(size_t)127;
    cpx<T>* W1 = reinterpret_cast<cpx<T>*>(sm + off);         // PP x C x CS: S/T, then g
    cpx<T>* W2 = W1 + PP * WP;                                // PP x C x CS: sources (2 spheres x NR x 2 modes), then a'
    cpx<T>* ACC = W2 + PP * WP;                               // NSLOT x NR x 2 modes x CS

    const int tid = threadIdx.x;
    if (tid == 0) {
        // (n, k) rows with the longest first so the work of a phase spreads evenly
        int e = 0;
        for (int n = L; n >= 1; n--)
            for (int k = 0; k <= n; k++) tabS[e++] = make_short2((short)n, (short)k);
        e = 0;
        for (int n = 1; n <= L; n++)
            for (int m = 1; m <= n; m++) tabQ[e++] = make_short2((short)n, (short)m);
        e = 0;
        for (int m = 0; m <= L; m++) {
            int m1 = m < 1 ? 1 : m;
            for (int line = m1; line <= L; line++) tabC[e++] = make_short2((short)m, (short)line);
        }
    }
    for (int e = tid; e < NSLOT * NR * 2 * CS; e += NT) ACC[e] = mk((T)0, (T)0);
    if (tid == 0) {
        mb_init(&bar[0], 1);
        mb_init(&bar[1], 1);
        mb_init(&bar[2], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int G = gridDim.x;
    const int NI = a.ntiles * a.nchunk;   // work items (tile, chunk), chunk fastest
    int tcur = blockIdx.x;
    if (tcur >= NI) return;
    auto tile_of = [&](int it) { return it / a.nchunk; };
    auto col0 = [&](int it) { return (size_t)(it % a.nchunk) * NR * (size_t)a.ld; };
    // output slots of pair qq of work item it
    auto slots_of = [&](int qq, int it, int& s_i, int& s_j) {
        if (a.pslot) {
            const short2 ps = a.pslot[qq];
            s_i = ps.x;
            s_j = ps.y;
        } else {
            const int4 ti = a.tiles[tile_of(it)];
            const int2 pr = a.pairs[qq];
            s_i = pr.x - (ti.z >> 16);
            s_j = ti.w ? (pr.y - (ti.z >> 16)) : (B + pr.y - (ti.z & 0xffff));
        }
    };
    // pairs of the step that starts at pair qq: two when the next pair of the
    // tile writes other slots
    auto step_np = [&](int qq, int it) -> int {
        if (PP == 1) return 1;
        const int4 ti = a.tiles[tile_of(it)];
        if (qq + 1 >= ti.x + ti.y) return 1;
        int a1, b1, a2, b2;
        slots_of(qq, it, a1, b1);
        slots_of(qq + 1, it, a2, b2);
        return (a1 != a2 && a1 != b2 && b1 != a2 && b1 != b2) ? 2 : 1;
    };
    // thread 0's iterators: operators two steps ahead, sources one step ahead
    int pf_t = tcur, pf_q = a.tiles[tile_of(tcur)].x;
    bool pf_ok = true;
    auto pf_adv = [&]() {
        pf_q += step_np(pf_q, pf_t);
        const int4 ti = a.tiles[tile_of(pf_t)];
        if (pf_q >= ti.x + ti.y) {
            pf_t += G;
            if (pf_t >= NI) { pf_ok = false; return; }
            pf_q = a.tiles[tile_of(pf_t)].x;
        }
    };
    auto load_ops = [&](int bb) {
        const int np_ = step_np(pf_q, pf_t);
        mb_expect(&bar[bb], (uint32_t)np_ * RECB);
        bulk_copy(opb + (size_t)bb * PP * REC, a.ops + (size_t)pf_q * REC, (uint32_t)np_ * RECB, &bar[bb]);   // consecutive records
        pf_adv();
    };
    auto load_sources = [&](int qq, int it) {
        const int np_ = step_np(qq, it);
        const cpx<T>* xs = a.x + col0(it);
        mb_expect(&bar[2], (uint32_t)np_ * 2u * NR * XB);
        for (int u = 0; u < np_; u++) {
            const int2 pr = a.pairs[qq + u];
            cpx<T>* w = W2 + (size_t)u * WP;
            for (int r = 0; r < NR; r++) {
                const cpx<T>* sj = xs + (size_t)r * a.ld + tile_sphere_base<SO>(a, pr.y, NB);   // source of j -> i
                const cpx<T>* si = xs + (size_t)r * a.ld + tile_sphere_base<SO>(a, pr.x, NB);   // source of i -> j
                if (CS == NB2) {   // both modes' columns in one copy
                    bulk_copy(w + (size_t)(0 * NR + r) * NB, sj, XB, &bar[2]);
                    bulk_copy(w + (size_t)(1 * NR + r) * NB, si, XB, &bar[2]);
                } else {           // a copy per mode, columns CS apart
                    for (int pm2 = 0; pm2 < 2; pm2++) {
                        bulk_copy(w + (size_t)((0 * NR + r) * 2 + pm2) * CS, sj + (size_t)pm2 * NB2, XB2, &bar[2]);
                        bulk_copy(w + (size_t)((1 * NR + r) * 2 + pm2) * CS, si + (size_t)pm2 * NB2, XB2, &bar[2]);
                    }
                }
            }
        }
    };
    if (tid == 0) {
        load_sources(pf_q, tcur);
        for (int bb = 0; bb < 2 && pf_ok; bb++) load_ops(bb);
    }
    int q = a.tiles[tile_of(tcur)].x;
    int t = 0;
    while (true) {
        const int4 tinfo = a.tiles[tile_of(tcur)];
        const int i0 = tinfo.z >> 16, j0 = tinfo.z & 0xffff;   // block starts
        const int diag = tinfo.w;
        const int b = t & 1;
        const int np = step_np(q, tcur);
        if (!mb_wait(&bar[b], (t >> 1) & 1) || !mb_wait(&bar[2], t & 1)) {
            if (tid == 0) atomicExch(a.err, MSTMG_ERR_CUDA);
            mb_wait(&bar[b ^ 1], ((t + 1) >> 1) & 1);
            mb_wait(&bar[2], t & 1);
            return;
        }
        int si[PP], sj[PP];
#pragma unroll
        for (int u = 0; u < PP; u++) {
            si[u] = 0;
            sj[u] = 0;
            if (u < np) slots_of(q + u, tcur, si[u], sj[u]);
        }
        if (tid < np) {
            const T* rec = opb + ((size_t)b * PP + tid) * REC;
            cpx<T> ep = mk(rec[0], rec[1]);
            cpx<T>* e = ephm + (size_t)tid * (2 * L + 1) + L;
            e[0] = mk((T)1, (T)0);
#pragma unroll
            for (int m = 1; m <= L; m++) {
                e[m] = ep * e[m - 1];
                e[-m] = cj(e[m]);
            }
        }
        __syncthreads();

        // ---- A: shift, phase, even/odd split of the staged sources.  Each
        //      thread takes IA items; all their loads are issued before any
        //      arithmetic, so the shared-memory latencies overlap ----
        {
            constexpr int NA1 = C * NS, NA = PP * NA1, IA = (NA + NT - 1) / NT;
            cpx<T> U[IA], V[IA], EU[IA];
            int sdst[IA], tdst[IA], mm[IA];   // S and T slots; m, with the shift flag as -m-1
#pragma unroll
            for (int k = 0; k < IA; k++) {
                const int idx = tid + k * NT;
                sdst[k] = -1;
                const int u = idx / NA1, li = idx - u * NA1;
                if (idx < NA && u < np) {
                    const int c = li / NS, jj = li - c * NS;
                    const short2 nm = tabS[jj];
                    const int n = nm.x, m = nm.y;
                    const int r = (c >> 1) % NR, dir = (c >> 1) / NR;
                    const bool swp = (dir != (int)((a.contran >> r) & 1u));
                    const cpx<T>* xs = W2 + (size_t)u * WP + (size_t)c * CS;
                    const cpx<T>* e = ephm + (size_t)u * (2 * L + 1) + L;
                    const int hp = hidx<L>(m, n), hm = m ? hidx<L>(-m, n) : hp;
                    // with the shift the +m and -m sources trade places (and take the sign (-1)^m)
                    U[k] = xs[swp ? hm : hp];
                    V[k] = xs[swp ? hp : hm];
                    EU[k] = e[dir ? -m : m];
                    sdst[k] = u * WP + c * CS + sofs(n) + m;
                    tdst[k] = u * WP + c * CS + NS + tofs(n) + m - 1;
                    mm[k] = swp ? -m - 1 : m;
                }
            }
#pragma unroll
            for (int k = 0; k < IA; k++) {
                if (sdst[k] < 0) continue;
                const bool swp = mm[k] < 0;
                const int m = swp ? -mm[k] - 1 : mm[k];
                if (m == 0) {
                    W1[sdst[k]] = (T)2 * U[k];
                } else {
                    const T sg = (m & 1) ? (T)-1 : (T)1;
                    const T s2 = swp ? sg : (T)1;
                    const cpx<T> uu = (s2 * U[k]) * EU[k], vv = (s2 * V[k]) * cj(EU[k]);
                    W1[sdst[k]] = uu + sg * vv;
                    W1[tdst[k]] = uu - sg * vv;
                }
            }
        }
        __syncthreads();

        // ---- B: forward rotation: a'(k) = P+Q, a'(-k) = (-1)^k (P-Q),
        //      P = E_n[k][:] s, Q = O_n[k][:] t ----
        for (int idx = tid; idx < np * NS * NG; idx += NT) {
            const int u = idx / (NS * NG), li = idx - u * (NS * NG);
            const int jj = li / NG, g = li - jj * NG;
            const short2 nk = tabS[jj];
            const int n = nk.x, k = nk.y;
            const T* rec = opb + ((size_t)b * PP + u) * REC;
            const T* Er = rec + 2 + op_rot_offset(n, L) + k * (n + 1);
            const T* Or = rec + 2 + op_rot_offset(n, L) + (n + 1) * (n + 1) + (k - 1) * n;
            T er[L + 1], orr[L];
#pragma unroll
            for (int mm = 0; mm <= L; mm++) er[mm] = (mm <= n) ? Er[mm] : (T)0;
#pragma unroll
            for (int mm = 0; mm < L; mm++) orr[mm] = (k >= 1 && mm < n) ? Or[mm] : (T)0;
#pragma unroll
            for (int cc = 0; cc < CB; cc++) {
                const int c = g * CB + cc;
                const cpx<T>* sv = W1 + u * WP + c * CS + sofs(n);
                const cpx<T>* tv = W1 + u * WP + c * CS + NS + tofs(n);
                cpx<T> P = mk((T)0, (T)0), Q = mk((T)0, (T)0);
#pragma unroll
                for (int mm = 0; mm <= L; mm++)
                    if (mm <= n) P = mac_r(P, er[mm], sv[mm]);
#pragma unroll
                for (int mm = 0; mm < L; mm++)
                    if (mm < n) Q = mac_r(Q, orr[mm], tv[mm]);
                cpx<T>* ap = W2 + u * WP + c * CS;
                if (k == 0) {
                    ap[hidx<L>(0, n)] = P;
                } else {
                    const T sk = (k & 1) ? (T)-1 : (T)1;
                    ap[hidx<L>(k, n)] = P + Q;
                    ap[hidx<L>(-k, n)] = sk * (P - Q);
                }
            }
        }
        __syncthreads();

        // ---- C: axial translation per degree m.  One item = one (m, line,
        //      direction, rhs): rows (j -> i) or columns (i -> j) of Z_m[0] and
        //      Z_m[1] applied to both modes, written as the back rotation's
        //      inputs s'(m) = g(m) + (-1)^m g(-m), t'(m) = g(m) - (-1)^m g(-m)
        //      (s'(0) = g(0)) in the packed S/T layout of W1 ----
        for (int idx = tid; idx < np * NS * 2 * NR; idx += NT) {
            const int u = idx / (NS * 2 * NR), li = idx - u * (NS * 2 * NR);
            const int zr = li / (2 * NR), dr = li - zr * (2 * NR);
            const int dir = dr / NR, r = dr - dir * NR;
            const short2 ml = tabC[zr];
            const int m = ml.x, line = ml.y;
            const int m1 = m < 1 ? 1 : m;
            const int dim = L - m1 + 1;
            const T* rec = opb + ((size_t)b * PP + u) * REC;
            const T* z0 = rec + 2 + RS + 2 * op_z_offset(m, L, L) + (dir ? 2 * (line - m1) : 2 * (line - m1) * dim);
            const T* z1 = z0 + 2 * dim * dim;
            const int zst = dir ? 2 * dim : 2;
            const cpx<T>* a0 = W2 + u * WP + (((dir * NR) + r) * 2 + 0) * CS;
            const cpx<T>* a1 = W2 + u * WP + (((dir * NR) + r) * 2 + 1) * CS;
            cpx<T>* o0 = W1 + u * WP + (((dir * NR) + r) * 2 + 0) * CS;
            cpx<T>* o1 = W1 + u * WP + (((dir * NR) + r) * 2 + 1) * CS;
            if (m == 0) {
                cpx<T> g0 = mk((T)0, (T)0), g1 = mk((T)0, (T)0);
                for (int v = 0; v < dim; v++) {
                    const cpx<T> z = mk(z0[v * zst], z0[v * zst + 1]);
                    const int h = (L + 2) * v;   // hidx(0, 1+v)
                    g0 = mac_c(g0, z, a0[h]);
                    g1 = mac_c(g1, z, a1[h]);
                }
                o0[sofs(line)] = g0;
                o1[sofs(line)] = g1;
            } else {
                cpx<T> gp0 = mk((T)0, (T)0), gm0 = gp0, gp1 = gp0, gm1 = gp0;
                const int hp0 = hidx<L>(m, m1), hm0 = hidx<L>(-m, m1);
                for (int v = 0; v < dim; v++) {
                    const cpx<T> za = mk(z0[v * zst], z0[v * zst + 1]);
                    const cpx<T> zb = mk(z1[v * zst], z1[v * zst + 1]);
                    const int hp = hp0 + (L + 2) * v, hm = hm0 + v;
                    gp0 = mac_c(gp0, za, a0[hp]);   // mode 0, +m: Z_m[0]
                    gm0 = mac_c(gm0, zb, a0[hm]);   // mode 0, -m: Z_m[1]
                    gp1 = mac_c(gp1, zb, a1[hp]);   // mode 1, +m: Z_m[1]
                    gm1 = mac_c(gm1, za, a1[hm]);   // mode 1, -m: Z_m[0]
                }
                const T sg = (m & 1) ? (T)-1 : (T)1;
                const int so = sofs(line) + m, to = NS + tofs(line) + m - 1;
                o0[so] = gp0 + sg * gm0;
                o0[to] = gp0 - sg * gm0;
                o1[so] = gp1 + sg * gm1;
                o1[to] = gp1 - sg * gm1;
            }
        }
        __syncthreads();

        // ---- the next step's sources stream into W2 while D runs ----
        if (tid == 0) {
            int nq = q + np, nit = tcur;
            bool have = true;
            if (nq >= tinfo.x + tinfo.y) {
                nit = tcur + G;
                if (nit < NI) nq = a.tiles[tile_of(nit)].x;
                else have = false;
            }
            if (have) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                load_sources(nq, nit);
            }
        }

        // ---- D: back rotation g'(k) = sum_m s'(m) E_n[m][k] +/- sum_m t'(m) O_n[m][k],
        //      phase, shift, accumulate into the tile's smem outputs (the
        //      pairs of a step write disjoint slots) ----
        for (int idx = tid; idx < np * NS * NG; idx += NT) {
            const int u = idx / (NS * NG), li = idx - u * (NS * NG);
            const int jj = li / NG, g = li - jj * NG;
            const short2 nk = tabS[jj];
            const int n = nk.x, k = nk.y;
            const T* rec = opb + ((size_t)b * PP + u) * REC;
            const T* E = rec + 2 + op_rot_offset(n, L);
            const T* O = E + (n + 1) * (n + 1);
            const cpx<T>* e = ephm + (size_t)u * (2 * L + 1) + L;
            T ec[L + 1], oc[L];
#pragma unroll
            for (int mm = 0; mm <= L; mm++) ec[mm] = (mm <= n) ? E[mm * (n + 1) + k] : (T)0;
#pragma unroll
            for (int mm = 0; mm < L; mm++) oc[mm] = (mm < n && k >= 1) ? O[mm * n + (k - 1)] : (T)0;
#pragma unroll
            for (int cc = 0; cc < CB; cc++) {
                const int c = g * CB + cc;
                const int p = c & 1, r = (c >> 1) % NR, dir = (c >> 1) / NR;
                const cpx<T>* sv = W1 + u * WP + c * CS + sofs(n);
                const cpx<T>* tv = W1 + u * WP + c * CS + NS + tofs(n);
                cpx<T> P = mk((T)0, (T)0), Q = mk((T)0, (T)0);
#pragma unroll
                for (int mm = 0; mm <= L; mm++)
                    if (mm <= n) P = mac_r(P, ec[mm], sv[mm]);
#pragma unroll
                for (int mm = 0; mm < L; mm++)
                    if (mm < n) Q = mac_r(Q, oc[mm], tv[mm]);
                const int slot = dir ? (u == 0 ? sj[0] : sj[PP - 1]) : (u == 0 ? si[0] : si[PP - 1]);
                cpx<T>* acc = ACC + ((slot * NR + r) * 2 + p) * CS;
                if (k == 0) {
                    acc[hidx<L>(0, n)] = acc[hidx<L>(0, n)] + (T)2 * P;
                } else {
                    const T sk = (k & 1) ? (T)-1 : (T)1;
                    const int im = dir ? -k : k;
                    cpx<T> outk = (P + Q) * e[-im];
                    cpx<T> outmk = (sk * (P - Q)) * e[im];
                    const bool swp = (dir != (int)((a.contran >> r) & 1u));
                    if (swp) { cpx<T> tt = outk; outk = sk * outmk; outmk = sk * tt; }
                    acc[hidx<L>(k, n)] = acc[hidx<L>(k, n)] + outk;
                    acc[hidx<L>(-k, n)] = acc[hidx<L>(-k, n)] + outmk;
                }
            }
        }
        __syncthreads();

        // ---- refill this operator buffer with the step after next ----
        if (tid == 0 && pf_ok) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            load_ops(b);
        }
        // ---- end of tile: flush the tile's outputs with coalesced atomics ----
        const bool last = (q + np == tinfo.x + tinfo.y);
        if (last) {
            cpx<T>* yc = a.y + col0(tcur);
            for (int idx = tid; idx < NSLOT * NR * NB; idx += NT) {
                const int slot = idx / (NR * NB);
                const int rem = idx - slot * (NR * NB);
                const int r = rem / NB, el = rem - r * NB;
                int ai = idx;   // CS == NB2: the accumulators in flush order
                if constexpr (CS != NB2) {
                    const int pe = el >= NB2 ? 1 : 0;
                    ai = ((slot * NR + r) * 2 + pe) * CS + (el - pe * NB2);
                }
                // grouped tiles carry their sphere-list row in z
                const int sph = a.tsph ? a.tsph[(size_t)tinfo.z * NSLOT + slot] : ((slot < B) ? (i0 + slot) : (j0 + slot - B));
                if (a.tsph ? sph >= 0 : (!(diag && slot >= B) && sph < a.nsph)) {
                    cpx<T> v = ACC[ai];
                    red_add<T>(yc + (size_t)r * a.ld + tile_sphere_base<SO>(a, sph, NB) + el, v);
                }
                ACC[ai] = mk((T)0, (T)0);
            }
            __syncthreads();
            tcur += G;
            if (tcur >= NI) break;
            q = a.tiles[tile_of(tcur)].x;
        } else {
            q += np;
        }
        t++;
    }
}

template <typename T, int L, int NR, int B, int PP> static size_t tiled_smem()
{
    constexpr int NS = L * (L + 3) / 2, NQ = L * (L + 1) / 2, CS = tiled_cs<T>(L), C = 4 * NR;
    size_t off = 64 + sizeof(short2) * (NS + NQ + NS);
    off = (off + 127) & ~(size_t)127;
    off += sizeof(cpx<T>) * PP * (2 * L + 1);
    off = (off + 127) & ~(size_t)127;
    off += sizeof(T) * 2 * PP * op_record_units(L, L);
    off = (off + 127) & ~(size_t)127;
    off += sizeof(cpx<T>) * ((size_t)2 * PP * C * CS + (size_t)2 * B * NR * 2 * CS);
    return off;
}

template <typename T, int L, int NR, int B, int PP, int MB> static int launch_mb(const TiledArgs<T>& a, int nsm, cudaStream_t st)
{
    size_t smem = tiled_smem<T, L, NR, B, PP>();
    if (smem > 227 * 1024) return -1;
    auto kern = a.soff ? translate_tiled_kernel<T, L, NR, B, PP, true, MB> : translate_tiled_kernel<T, L, NR, B, PP, false, MB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = (int)((228 * 1024) / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    if (per_sm > MB) per_sm = MB;
    if (a.ctas_per_sm >= 1 && a.ctas_per_sm < per_sm) per_sm = a.ctas_per_sm;
    int blocks = nsm * per_sm;
    if (blocks > a.ntiles * a.nchunk) blocks = a.ntiles * a.nchunk;
    if (blocks < 1) return 0;
    kern<<<blocks, 256, smem, st>>>(a);
    launch_counter() += 1;
    return 0;
}

// FP64 passes of orders 5-7 whose work items do not fill one wave of three
// CTAs per SM run the two-CTA instance: with few CTAs the 128-register budget
// (no spills) is faster per CTA (20 spheres of order 7, FP64 solve: 3.59 ms
// with the three-CTA instance, 3.05 ms with this one)
template <typename T, int L, int NR, int B, int PP> static int launch_pp(const TiledArgs<T>& a, int nsm, cudaStream_t st)
{
    constexpr int MB = tiled_minb<T, L, NR, PP>();
    if constexpr (sizeof(T) == 8 && MB == 3) {
        if (a.ntiles * a.nchunk < 3 * nsm || (a.ctas_per_sm >= 1 && a.ctas_per_sm < 3))
            return launch_mb<T, L, NR, B, PP, 2>(a, nsm, st);
    }
    return launch_mb<T, L, NR, B, PP, MB>(a, nsm, st);
}

// Two pairs a step only when asked for (FP32 passes of one or two columns):
// it fills the rotation phases and halves the barriers per pair, but its
// shared memory leaves two CTAs per SM instead of three, and measured on the
// 500-sphere aggregate it is slower (FP32, 2 columns: 2.28 against 1.86 ms;
// 1 column: 1.82 against 1.40 ms).
template <typename T, int L, int NR, int B> static int launch_one(const TiledArgs<T>& a, int nsm, cudaStream_t st)
{
    if constexpr (sizeof(T) == 4 && NR <= 2) {
        if (a.pairs_per_step == 2) return launch_pp<T, L, NR, B, 2>(a, nsm, st);
    }
    return launch_pp<T, L, NR, B, 1>(a, nsm, st);
}

template <typename T, int L> static int launch_L(const TiledArgs<T>& a, int nsm, cudaStream_t st)
{
    switch (a.nrhs) {
    case 1: return launch_one<T, L, 1, TILE_B>(a, nsm, st);
    case 2: return launch_one<T, L, 2, TILE_B>(a, nsm, st);
    case 4:
        if constexpr (sizeof(T) == 8) return -1;   // FP64 with four columns: the generic kernel
        else return launch_one<T, L, 4, TILE_B>(a, nsm, st);
    default: return -1;
    }
}

template <typename T> int launch_translate_tiled(const TiledArgs<T>& a, int L, int nsm, cudaStream_t st)
{
    switch (L) {
    case 3: return launch_L<T, 3>(a, nsm, st);
    case 4: return launch_L<T, 4>(a, nsm, st);
    case 5: return launch_L<T, 5>(a, nsm, st);
    case 6: return launch_L<T, 6>(a, nsm, st);
    case 7: return launch_L<T, 7>(a, nsm, st);
    case 8: return launch_L<T, 8>(a, nsm, st);
    case 9: return launch_L<T, 9>(a, nsm, st);
    case 10: return launch_L<T, 10>(a, nsm, st);
    default: return -1;
    }
}
bool tiled_supported(int L, int nrhs) { return L >= 3 && L <= 10 && (nrhs == 1 || nrhs == 2 || nrhs == 4); }

template int launch_translate_tiled<double>(const TiledArgs<double>&, int, int, cudaStream_t);
template int launch_translate_tiled<float>(const TiledArgs<float>&, int, int, cudaStream_t);

// Self-test of the bounded wait: one CTA waits on an mbarrier whose
// transaction never arrives (an expected byte count with no copy issued), gives
// up after `limit` polls per thread and records MSTMG_ERR_CUDA in *err -- the
// path the translation kernel takes when a bulk copy does not complete.  No
// asynchronous operation is in flight when it returns.
__global__ void wait_selftest_kernel(int limit, int* err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mb_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) mb_expect(&bar, 16u);
    __syncthreads();
    if (!mb_wait(&bar, 0u, limit)) {
        if (threadIdx.x == 0) atomicExch(err, MSTMG_ERR_CUDA);
    }
}

int launch_wait_selftest(int limit, int* err, cudaStream_t st)
{
    wait_selftest_kernel<<<1, 64, 0, st>>>(limit, err);
    launch_counter() += 1;
    return 0;
}
