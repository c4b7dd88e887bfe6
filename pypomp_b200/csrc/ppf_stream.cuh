// ppf_stream.cuh -- the per-tile bodies of the streaming particle-filter
// kernels: initial states (init_tile), and resampling + propagation
// (resprop_tile).  ppf_pfilter.cu wraps them in one launch per step
// (k_init, k_resprop); the persistent MOP forward (ppf_mop.cu) calls the
// same bodies for its own tile between grid barriers, so both give
// bit-identical results.
#pragma once

#include "ppf_kernels.cuh"

namespace ppf {

// Initial states of tile b of filter f, propagated into observation 0.
template <class M, int TPB, bool INJ, bool FAST = false>
__device__ __forceinline__ void init_tile(const Args& a, int f, int b) {
  __shared__ typename M::Consts c;
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  constexpr int DX = M::MAXDX;
  const int u = filter_unit(a, f);
  load_consts<M>(a, f, c);
  __syncthreads();
  const typename M::Consts cr = c;
  Obs<M> ob;
  ob.load(a, u, 0);
  const int J = a.J;
  float* X = a.X[0] + (size_t)f * DX * J;
  float* W = a.W[0] + (size_t)f * J;
  float* logw = a.logw ? a.logw + ((size_t)f * a.T) * J : nullptr;
  const bool pm = (a.flags & PPF_F_PMEAN) != 0;
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  double px[DX];
#pragma unroll
  for (int d = 0; d < DX; ++d) px[d] = 0.0;
  const int j0 = b * a.tile;
  const int j1 = min(j0 + a.tile, J);
  const float base = (a.mode == MODE_MOP ? 0.0f : a.base_init);
  for (int k0 = j0 + 4 * threadIdx.x; k0 < j1; k0 += 4 * TPB) {
    float z0[4 * (M::NZ0 > 0 ? M::NZ0 : 1)];
    float z[4 * M::NZ];
    group_noise<M::NZ0, INJ, FAST>(a, f, 0, k0, z0);
    group_noise<M::NZ, INJ, FAST>(a, f, 1, k0, z);
    float xo[4][DX];
    float wo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float x[DX];
      M::rinit(cr, z0 + e * M::NZ0, x);
      if (a.mop_ckpt && k0 + e < j1)
#pragma unroll
        for (int d = 0; d < DX; ++d) a.mop_ckpt[((size_t)f * a.nseg * DX + d) * J + k0 + e] = x[d];
      wo[e] = base + step1<M>(cr, ob, x, z + e * M::NZ);
#pragma unroll
      for (int d = 0; d < DX; ++d) xo[e][d] = x[d];
      if (k0 + e < j1) {
        accum_maxmin(wo[e], mx, mn, nn);
        if (pm)
#pragma unroll
          for (int d = 0; d < DX; ++d) px[d] += (double)x[d];
      }
    }
    store_group<DX>(X, W, logw, J, k0, xo, wo, 0, min(4, j1 - k0));
  }
  block_maxmin_u32<TPB>(mx, mn, smk);
  nn = __syncthreads_or(nn);
  Acc* acc = a.acc[0] + f;
  if (threadIdx.x == 0) {
    atomicMax(&acc->maxkey, mx);
    atomicMin(&acc->minkey, mn);
    if (nn) atomicOr(&acc->nan, 1u);
    if (b == 0) a.loglik[f] = 0.0;
  }
  if (pm) {
#pragma unroll
    for (int d = 0; d < DX; ++d) {
      const double s = block_sum_f64<TPB>(px[d], sd);
      if (threadIdx.x == 0) atomicAdd(&acc->px[d], s);
    }
  }
}

// Resample the parents of one tile and propagate their children to the next
// observation (rproc + dmeas fused), writing the next step's X, W.
//   1. fixed-point weights of the tile's parents, block scan, plus the tile's
//      exclusive prefix from k_sum: the exact CDF of every parent;
//   2. closed-form first-child offset st[l] = nchild(C_{l-1}) per parent into
//      shared memory (st[l] = l on steps without resampling), parent states
//      staged in shared memory;
//   3. merge-path partition of the tile's children [st[0], st[n]) into TPB
//      near-equal chunks of whole groups: one binary search for a chunk's
//      first parent, then a linear walk; per group of 4 children one set of
//      Philox calls (every word used), rproc + dmeas, float4 stores.
// CTAs per SM the register budget is sized for (256-thread CTAs): 4 (64
// registers) for one-variable states and for 2-D states with two normals per
// child (measured on the 2-D LG batch: 4 CTAs per SM beat 3 by 7 %), else 3
// (80 registers; the SV kernel spills at 64).
template <class M>
struct RespropOccupancy {
  static constexpr int B = M::WIDE ? 1 : (M::MAXDX == 1 || (M::MAXDX == 2 && M::NZ == 2)) ? 4 : 3;
};

// The body for tile b of filter f at step t.  TMA: stage the tile's parent
// rows with bulk copies (the streaming kernel) or plain loads (the persistent
// MOP kernel, whose mbarriers would otherwise need a phase per step).
template <class M, int TPB, int IT, bool INJ, bool TMA, bool FAST = false>
__device__ __forceinline__ void resprop_tile(const Args& a, int t, int f, int b) {
  constexpr int TILE = TPB * IT;
  constexpr int DX = M::MAXDX;
  constexpr int RUN = IT;            // children per thread run: TPB runs cover a full tile
  static_assert(RUN % 4 == 0, "children are drawn in groups of 4");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* xs = reinterpret_cast<float*>(smem_raw);                              // [DX][TILE]
  int* st = reinterpret_cast<int*>(smem_raw + sizeof(float) * DX * TILE);      // [TILE + 1]
  float* wcar = reinterpret_cast<float*>(st + TILE + 4);                      // [TILE] (no-resample steps)
  float* wsm = wcar;                                                           // W row lands here first
  __shared__ __align__(8) uint64_t bar[2];                                     // [0]: W row, [1]: X rows
  __shared__ typename M::Consts c;
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];

  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  const int p = t & 1;
  // reset the next step's tile-total slot and done-count (before any early
  // exit: finished filters of a ragged panel still own these slots)
  if (threadIdx.x == 0) {
    a.desc[p ^ 1][(size_t)f * a.ntiles + b] = 0ull;
    if (b == 0 && f == 0) a.counter[p ^ 1] = 0;
    if (b == 0) a.fdone[p ^ 1][f] = 0u;   // the next step's tile count
  }
  if (t >= Tf) return;
  const Acc& acc = a.acc[p][f];   // read in place (a copy would sit in local memory)
  const uint64_t tot = a.tot[f];
  if (b == 0 && threadIdx.x == 0) finalize_step(a, f, t, acc, tot, a.loglik + f);
  const bool last = (t == Tf - 1);
  if (last && !a.anc) return;
  const int J = a.J;
  const int jt = b * TILE;
  const int ntile = min(TILE, J - jt);
  // Rows of this tile are contiguous: with J % 4 == 0 every row starts
  // 16-byte aligned and ntile is a multiple of 4, so one thread issues TMA
  // bulk copies of the W row and the DX state rows into shared memory; the
  // parent-phase arithmetic below overlaps the state copies.
  const bool bulk = TMA && (J & 3) == 0;
  const float* Wc = a.W[p] + (size_t)f * J;
  const float* Xc = a.X[p] + (size_t)f * DX * J;
  if (bulk) {
    if (threadIdx.x == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
      mbar_expect_tx(&bar[0], (uint32_t)(ntile * 4));
      bulk_g2s(wsm, Wc + jt, (uint32_t)(ntile * 4), &bar[0]);
      mbar_expect_tx(&bar[1], (uint32_t)(ntile * 4 * DX));
#pragma unroll
      for (int d = 0; d < DX; ++d) bulk_g2s(xs + d * TILE, Xc + (size_t)d * J + jt, (uint32_t)(ntile * 4), &bar[1]);
    }
  }
  load_consts<M>(a, f, c);
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = !nanf && Mx == -INFINITY;
  const bool rs = decide_resample(a, acc);
  float* Xn = a.X[p ^ 1] + (size_t)f * DX * J;
  float* Wn = a.W[p ^ 1] + (size_t)f * J;
  int* anc = a.anc ? a.anc + ((size_t)f * a.T + t) * J : nullptr;
  float* logw = a.logw ? a.logw + ((size_t)f * a.T + t + 1) * J : nullptr;
  const bool pm = (a.flags & PPF_F_PMEAN) != 0;
  Obs<M> ob;
  if (!last) ob.load(a, u, t + 1);
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  double px[DX];
#pragma unroll
  for (int d = 0; d < DX; ++d) px[d] = 0.0;
  const float base = (a.mode == MODE_MOP) ? 0.0f : a.base_rs;
  const int l0 = threadIdx.x * IT;
  __syncthreads();   // barrier init visible to all threads
  // A wait that gives up marks the call failed (error bit 1, PPF_ETIMEOUT) and
  // then still drains its own copy, so the CTA never leaves with a bulk copy
  // in flight into its shared memory; what it computes is flagged invalid.
  bool ok = true;
  if (bulk && !mbar_wait(&bar[0], 0, a.spin_cap)) {
    ok = false;
    mbar_wait(&bar[0], 0);
  }

  // 1-2. parents: CDF and first-child offsets (or identity), staged states
  {
    float wv[IT];
    if (bulk && l0 + IT <= ntile) {
#pragma unroll
      for (int i = 0; i < IT; i += 4) {
        const float4 v4 = *reinterpret_cast<const float4*>(wsm + l0 + i);
        wv[i] = v4.x; wv[i + 1] = v4.y; wv[i + 2] = v4.z; wv[i + 3] = v4.w;
      }
    } else if (bulk) {
#pragma unroll
      for (int i = 0; i < IT; ++i) wv[i] = (l0 + i < ntile) ? wsm[l0 + i] : 0.0f;
    } else {
#pragma unroll
      for (int i = 0; i < IT; ++i) wv[i] = (l0 + i < ntile) ? Wc[jt + l0 + i] : 0.0f;
    }
    if (rs) {
      const Offsets o = make_offsets(tot, resample_u32(a, f, t), J);
      const uint64_t E = a.excl[(size_t)f * a.ntiles + b];
      uint64_t q[IT];
#pragma unroll
      for (int i = 0; i < IT; ++i) q[i] = (l0 + i < ntile) ? qweight_from_e(wv[i]) : 0ull;   // k_sum left e
      // the exclusive prefix of this thread's run within the tile, from k_sum
      const uint64_t tex = a.runpre[((size_t)f * a.ntiles + b) * TPB + threadIdx.x];
      if (l0 < ntile && !run_has_heavy_e(wv, tot, J)) {
        OffWalk wk = offwalk_init(o, E + tex);
        st[l0] = wk.k;
#pragma unroll
        for (int i = 0; i < IT; ++i) {
          if (l0 + i >= ntile) break;
          const int kn = offwalk_add(o, wk, q[i]);
          if (i + 1 < IT || l0 + i + 1 == ntile) st[l0 + i + 1] = kn;
        }
      } else if (l0 < ntile) {
        uint64_t C = E + tex;   // a heavy parent in the run: closed form throughout
        st[l0] = nchild_fast(o, C);
#pragma unroll
        for (int i = 0; i < IT; ++i) {
          if (l0 + i >= ntile) break;
          C += q[i];
          const int kn = nchild_fast(o, C);
          if (i + 1 < IT || l0 + i + 1 == ntile) st[l0 + i + 1] = kn;
        }
      }
    } else {
      float lt32 = 0.0f;
      if (nanf) lt32 = __int_as_float(0x7fc00000);
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
      const float nwc = -pp_logf((float)J);
#pragma unroll
      for (int i = 0; i < IT; ++i)
        if (l0 + i < ntile) {
          st[l0 + i] = jt + l0 + i;
          wcar[l0 + i] = collapsed ? nwc : wv[i] - lt32;
        }
      if (l0 < ntile && l0 + IT >= ntile) st[ntile] = jt + ntile;
    }
  }
  if (bulk) {
    if (!mbar_wait(&bar[1], 0, a.spin_cap)) {
      ok = false;
      mbar_wait(&bar[1], 0);
    }
  } else {
    for (int l = threadIdx.x; l < ntile; l += TPB)
#pragma unroll
      for (int d = 0; d < DX; ++d) xs[d * TILE + l] = Xc[d * J + jt + l];
  }
  if (!ok && threadIdx.x == 0) atomicOr(a.err, 1u);
  __syncthreads();
  const typename M::Consts cr = c;
  const int klo = st[0], khi = st[ntile];
  // MOP: keep the first-child offsets of every parent for the adjoint sweep
  if (a.mop_off) {
    int* off = a.mop_off + ((size_t)f * a.T + t) * (J + 1) + jt;
    for (int l = threadIdx.x; l <= ntile; l += TPB)
      if (l < ntile || jt + ntile == J) off[l] = st[l];
  }
  // MOP: checkpoint the resampled states x^F_t when step t+1 opens a segment
  float* ckpt = nullptr;
  if (a.mop_ckpt && (t + 1) % a.ckpt_every == 0 && (t + 1) / a.ckpt_every < a.nseg)
    ckpt = a.mop_ckpt + ((size_t)f * a.nseg + (t + 1) / a.ckpt_every) * DX * J;

  // 3. children, drawn in Philox groups of G: the tile's groups are split into
  //    TPB contiguous, near-equal chunks (a tile's child count fluctuates around
  //    TILE; fixed-size runs left a second run to a few threads whenever it
  //    exceeded TILE, and the whole CTA waited for them)
  constexpr int G = ChildGroup<M::NZ>::G;
  static_assert((RUN % G) == 0 && (4 % G) == 0, "groups align with the 4-aligned start");
  const int kA = klo & ~3;
  const int ngr = (khi - kA + G - 1) / G;
  const int g0 = (int)(((long long)threadIdx.x * ngr) / TPB);
  const int g1 = (int)(((long long)(threadIdx.x + 1) * ngr) / TPB);
  if (g0 < g1) {
    const int ka = kA + G * g0;
    int l = find_parent(st, ntile, max(ka, klo));
#pragma unroll 1
    for (int g = 0; g < g1 - g0; ++g) {
      const int k0 = ka + G * g;
      if (k0 >= khi) break;
      const int lo = max(0, klo - k0), hi = min(G, khi - k0);   // valid e in [lo, hi)
      float z[G * M::NZ];
      if (!last) group_noise_g<G, M::NZ, INJ, FAST>(a, f, t + 2, k0, z);
      float xo[G][DX];
      float wo[G];
#pragma unroll
      for (int e = 0; e < G; ++e) {
        const int k = k0 + e;
        const bool valid = (e >= lo) & (e < hi);
        if (valid) {
          int adv = 0;
          while (l + 1 < ntile && st[l + 1] <= k) {
            ++l;
            if (++adv > 8) { l = find_parent(st, ntile, k); break; }
          }
          if (anc) anc[k] = jt + l;
        }
        float x[DX];
#pragma unroll
        for (int d = 0; d < DX; ++d) x[d] = xs[d * TILE + l];
        if (ckpt && valid)
#pragma unroll
          for (int d = 0; d < DX; ++d) ckpt[d * J + k] = x[d];
        const float wb = rs ? base : wcar[l];
        wo[e] = wb + step1<M>(cr, ob, x, z + e * M::NZ);
#pragma unroll
        for (int d = 0; d < DX; ++d) xo[e][d] = x[d];
        if (valid) {
          accum_maxmin(wo[e], mx, mn, nn);
          if (pm)
#pragma unroll
            for (int d = 0; d < DX; ++d) px[d] += (double)x[d];
        }
      }
      if (!last) store_group_g<G, DX>(Xn, Wn, logw, J, k0, xo, wo, lo, hi);
    }
  }
  if (last) return;
  block_maxmin_u32<TPB>(mx, mn, smk);
  nn = __syncthreads_or(nn);
  Acc* an = a.acc[p ^ 1] + f;
  if (threadIdx.x == 0) {
    if (mx) atomicMax(&an->maxkey, mx);
    if (mn != 0xffffffffu) atomicMin(&an->minkey, mn);
    if (nn) atomicOr(&an->nan, 1u);
  }
  if (pm) {
#pragma unroll
    for (int d = 0; d < DX; ++d) {
      const double s = block_sum_f64<TPB>(px[d], sd);
      if (threadIdx.x == 0) atomicAdd(&an->px[d], s);
    }
  }
}

}  // namespace ppf
