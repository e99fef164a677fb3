// riemann_exact.cu -- batched isolated exact Riemann solves with a learned
// initial guess for the star pressure, and the hand-written training of that
// guess (no counterpart in FLASH5, whose unsplit path only has approximate
// solvers, hy_getFaceFlux.F90:324-372).  The solver itself (Toro ch. 4) and
// the per-warp tensor-core network inference (mma.sync) live in
// exact_rs.cuh, shared with the hydro face fluxes; the batched solves and
// predictions run the network on the tcgen05 tensor cores by default
// (k_solve_tc, primitives in tc05.cuh).
//
// Learned path: Newton gets three evaluations from the network's guess; if
// that does not converge, the solve restarts from the two-rarefaction guess
// (fallback), so the converged p* never depends on the network.
//
// Training: hand-written FP32 forward/backward kernels (mean-squared error
// on ln(p*/p_TR)) and an Adam update, on interface states harvested from
// the solver's own runs (isolated solves or hydro face states).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../../include/flash_hy.h"
#include "exact_rs.cuh"
#include "tc05.cuh"

namespace rx {

using namespace xrs;

// ---------------------------------------------------------------------------
// isolated solves: states[7][n] = (dl, ul, pl, dr, ur, pr, gamma)
// out[2][n] = (p*, u*); iters[n] = Newton evaluations (incl. fallback);
// flags bit0: fell back to the two-rarefaction guess, bit1: vacuum,
// bit2: not converged
// ---------------------------------------------------------------------------
constexpr int SOLVE_THREADS = 256;

__device__ __forceinline__ void load_state(const double *__restrict__ S, long n, long i, Side &L, Side &R, Gas &G) {
  L.d = S[i]; L.u = S[n + i]; L.p = S[2 * n + i];
  R.d = S[3 * n + i]; R.u = S[4 * n + i]; R.p = S[5 * n + i];
  const double g = S[6 * n + i];
  G = gas_of(g);
  L.c = sqrt(g * L.p / L.d); R.c = sqrt(g * R.p / R.d);
  L.w = powp(L.p, G.z); R.w = powp(R.p, G.z);
}

// the state of pair i, or a harmless placeholder for a lane past the end
// (lanes of the last tile take part in the warp and CTA collectives)
__device__ __forceinline__ void load_or_dummy(const double *__restrict__ S, long n, long i, bool valid, Side &L,
                                              Side &R, Gas &G) {
  if (valid) {
    load_state(S, n, i, L, R, G);
  } else {
    G = gas_of(1.4);
    L.d = R.d = 1.0; L.u = R.u = 0.0; L.p = R.p = 1.0; L.c = R.c = sqrt(1.4); L.w = R.w = 1.0;
  }
}

// Newton from w0 (three evaluations where the network gave the start, else
// max_iter) and the recording of the result; returns true where a network
// start did not converge, so that the pair is queued for k_fallback
__device__ __forceinline__ bool solve_store(const Side &L, const Side &R, const SideK &kl, const SideK &kr,
                                            const Gas &G, bool vac, bool net, double w0, double tol, int max_iter,
                                            bool valid, long i, long n, double *__restrict__ out,
                                            unsigned char *__restrict__ iters, unsigned char *__restrict__ flags,
                                            unsigned &st) {
  unsigned char fl = net ? 8 : 0;
  int its = 0;
  bool pending = false;
  Star S{0.0, 0.5 * (L.u + R.u), 0.0};
  if (vac) {
    fl |= 2;
  } else {
    int k = newton(L, R, kl, kr, G, w0, tol, net ? 3 : max_iter, S);
    if (k > 0) its = k;
    else if (net) pending = true;
    else { its = max_iter; fl |= 4; st |= FLASH_HY_ERR_NEWTON_NOCONV; }
  }
  if (valid && !pending) {
    out[i] = S.p; out[n + i] = S.u;
    if (iters) iters[i] = (unsigned char)(its > 255 ? 255 : its);
    if (flags) flags[i] = fl;
  }
  return pending;
}

// append the warp's pending lanes to the fallback queue (one atomic per warp)
__device__ __forceinline__ void enqueue(bool pending, long i, int *queue, int *qcount) {
  const int lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(0xffffffffu, pending);
  if (m) {
    int base_q = 0;
    if (lane == __ffs(m) - 1) base_q = atomicAdd(qcount, __popc(m));
    base_q = __shfl_sync(0xffffffffu, base_q, __ffs(m) - 1);
    if (pending) queue[base_q + __popc(m & ((1u << lane) - 1))] = (int)i;
  }
}

// learned != 0: Newton gets three evaluations from the network's guess where
// the network is consulted (strong waves, inexact two-rarefaction guess;
// elsewhere the two-rarefaction start with the full iteration budget);
// lanes that have not converged are appended to `queue` (warp-aggregated
// atomics) and re-solved from the two-rarefaction guess by k_fallback, so no
// warp waits for a fallback lane.  Here the network runs per warp on
// mma.sync (mlp_lane); k_solve_tc below is the tcgen05 form.
// One instantiation per path, so that the two-rarefaction path does not
// carry the network's register footprint.
template <bool learned>
__global__ void __launch_bounds__(SOLVE_THREADS, learned ? 2 : 1)
k_solve(const double *__restrict__ S, long n, double *__restrict__ out, unsigned char *__restrict__ iters,
        unsigned char *__restrict__ flags, const MlpPacked *__restrict__ w, double tol, int max_iter, int *queue,
        int *qcount, unsigned *status) {
  __shared__ __align__(16) MlpPacked M;
  if (learned) { load_packed(M, w); __syncthreads(); }
  const long stride = (long)gridDim.x * blockDim.x;
  unsigned st = 0;
  // grid-stride loop whose trip count is uniform across a warp
  for (long base = (long)blockIdx.x * blockDim.x; base < n; base += stride) {
    const long i = base + threadIdx.x;
    const bool valid = i < n;
    Side L, R;
    Gas G;
    load_or_dummy(S, n, i, valid, L, R, G);
    const SideK kl = side_k(L, G), kr = side_k(R, G);
    const bool vac = vacuum(L, R, G);
    const double wtr = vac ? 0.0 : tr_w(L, R, kl, kr, G);
    const double ptr = vac ? 0.0 : p_of_w(wtr, G);
    double w0 = wtr;
    bool net = false;
    if (learned) {
      // the network is consulted for strong waves with an inexact
      // two-rarefaction guess; warps without such a lane skip it
      net = valid && !vac && !tr_exact(L, R, ptr) && strong_waves(L, R);
      if (__any_sync(0xffffffffu, net)) {
        float f[NIN];
        if (net) features(L, R, G.g, ptr, f);
        else for (int k = 0; k < NIN; ++k) f[k] = 0.f;
        float y = fminf(fmaxf(mlp_lane(M, f), -20.f), 20.f);
        if (net) w0 = wtr * (double)expf(float(G.z) * y);    // (p*/p_TR)^z
      }
    }
    const bool pending = solve_store(L, R, kl, kr, G, vac, net, w0, tol, max_iter, valid, i, n, out, iters, flags, st);
    if (learned) enqueue(pending && valid, i, queue, qcount);
  }
  if (st) atomicOr(status, st);
}

// ---------------------------------------------------------------------------
// The learned path with the network on the fifth-generation tensor cores.
// A CTA of 128 threads takes tiles of 128 pairs (one per thread, grid-stride
// over tiles).  Where any pair of the tile consults the network, thread m
// writes row m of the tile's feature matrix to shared memory and one thread
// issues the three layers as tcgen05.mma with the accumulator in TMEM:
//   layer 1  [128 x 16] x [16 x 64]: K holds the 8 features, then 1, 1
//            against the bias split into BF16 high and low parts;
//   layer 2  [128 x 80] x [80 x 64]: K holds the 64 hidden units, then 1, 1
//            against the bias's two parts;
//   layer 3  [128 x 64] x [64 x 16]: N column 0 the BF16 high part of w3,
//            column 1 its low part, y = D[m][0] + D[m][1] + b3.
// Between the layers each thread reads its row back (tcgen05.ld), and one
// cvt.rn.relu.bf16x2 per two units gives the BF16 operands of the next
// layer.  The BF16 operands, FP32 accumulation and the weights are those of
// mlp_lane; the FP32 biases and w3 enter as two BF16 parts (16 significant
// bits) and the accumulation order differs, so the output agrees with
// mlp_lane to that rounding.  SOLVE = false writes the network's output
// for every pair (0 for vacuum) instead of solving.
//
// Waits on the MMA completions are bounded (about a second of SM clocks);
// a CTA that gives up sets FLASH_HY_ERR_TIMEOUT, waits (bounded) for the MMA
// in flight, frees its TMEM and leaves.
// ---------------------------------------------------------------------------
constexpr int TC_THREADS = 128;
constexpr uint32_t TC_TMEM_COLS = 64;           // one 128 x 64 FP32 accumulator, reused by the three layers
constexpr long long kTcWaitCycles = 1LL << 31;
constexpr int kK1 = 16, kK2 = NH + 16;          // padded K of layers 1 and 2
constexpr uint32_t kLbo = 128;                  // core matrices along K
constexpr uint32_t kSboA1 = kK1 / 8 * 128, kSboA2 = kK2 / 8 * 128, kSboW3 = NH / 8 * 128;

struct __align__(128) TcSmem {
  uint8_t X[128 * kK2 * 2];                     // the tile's A operand: features, then hidden rows of layer 2, of layer 3
  uint8_t W2[NH * kK2 * 2];                     // [n][k]: W2, then b2 high, b2 low
  uint8_t W1[NH * kK1 * 2];                     // [n][k]: W1, then b1 high, b1 low
  uint8_t W3[16 * NH * 2];                      // [n][k]: n = 0 w3 high, n = 1 w3 low, others 0
  float b3;
  uint32_t tmem_base;
  int fail;
  unsigned long long bar;
};

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
__device__ __forceinline__ uint32_t bf16_bits(__nv_bfloat16 v) { return (uint32_t)__bfloat16_as_ushort(v); }
// {relu(lo), relu(hi)} rounded to BF16, lo in the low half
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;\n" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

// Five CTAs per SM for the solve (96 registers, a few spilled), six for
// the network alone (80): measured on 1e8 pairs, 11.1 -> 10.5 ms and
// 5.6 -> 5.4 ms against four.
template <bool SOLVE>
__global__ void __launch_bounds__(TC_THREADS, SOLVE ? 5 : 6)
k_solve_tc(const double *__restrict__ S, long n, double *__restrict__ out, unsigned char *__restrict__ iters,
           unsigned char *__restrict__ flags, const MlpPacked *__restrict__ w, double tol, int max_iter, int *queue,
           int *qcount, unsigned *status, float *__restrict__ yout) {
  __shared__ TcSmem sm;
  const int t = threadIdx.x, wid = t >> 5;
  const uint4 ones = make_uint4(0x3F803F80u, 0u, 0u, 0u);      // BF16 1.0, 1.0, then zeros
  {
    // weights into the canonical layouts (16-byte chunks of 8 values along K)
    const uint4 *W1g = reinterpret_cast<const uint4 *>(&w->W1[0][0]);
    const uint4 *W2g = reinterpret_cast<const uint4 *>(&w->W2[0][0]);
    if (t < NH) {
      __nv_bfloat16 h1, l1, h2, l2;
      split_bf16(w->b1[t], h1, l1);
      split_bf16(w->b2[t], h2, l2);
      *reinterpret_cast<uint4 *>(sm.W1 + tc05::canon_off(t, 0, kSboA1)) = W1g[2 * t];
      *reinterpret_cast<uint4 *>(sm.W1 + tc05::canon_off(t, 1, kSboA1)) =
          make_uint4(bf16_bits(h1) | (bf16_bits(l1) << 16), 0u, 0u, 0u);
      *reinterpret_cast<uint4 *>(sm.W2 + tc05::canon_off(t, 8, kSboA2)) =
          make_uint4(bf16_bits(h2) | (bf16_bits(l2) << 16), 0u, 0u, 0u);
      *reinterpret_cast<uint4 *>(sm.W2 + tc05::canon_off(t, 9, kSboA2)) = make_uint4(0u, 0u, 0u, 0u);
    }
    for (int q = t; q < NH * NH / 8; q += TC_THREADS)
      *reinterpret_cast<uint4 *>(sm.W2 + tc05::canon_off(q >> 3, q & 7, kSboA2)) = W2g[q];
    // W3: 16 rows x 8 chunks; thread t fills chunk t & 7 of row t >> 3
    {
      const int row = t >> 3, c = t & 7;
      uint32_t v[4] = {0u, 0u, 0u, 0u};
      if (row < 2) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          __nv_bfloat16 ha, la, hb, lb;
          split_bf16(w->w3[8 * c + 2 * e], ha, la);
          split_bf16(w->w3[8 * c + 2 * e + 1], hb, lb);
          v[e] = row == 0 ? (bf16_bits(ha) | (bf16_bits(hb) << 16)) : (bf16_bits(la) | (bf16_bits(lb) << 16));
        }
      }
      *reinterpret_cast<uint4 *>(sm.W3 + tc05::canon_off(row, c, kSboW3)) = make_uint4(v[0], v[1], v[2], v[3]);
    }
    if (t == 0) { sm.b3 = w->b3; sm.fail = 0; }
  }
  if (t == 0) tc05::mbar_init(&sm.bar, 1);
  if (wid == 0) tc05::tmem_alloc(&sm.tmem_base, TC_TMEM_COLS);
  tc05::fence_smem_to_async();
  tc05::fence_before_sync();
  __syncthreads();
  tc05::fence_after_sync();
  const uint32_t tmem = sm.tmem_base;
  const uint32_t trow = tmem + ((uint32_t)(wid * 32) << 16);       // this warp's TMEM lanes
  const uint32_t xs = tc05::smem_addr(sm.X);
  const uint32_t w1s = tc05::smem_addr(sm.W1), w2s = tc05::smem_addr(sm.W2), w3s = tc05::smem_addr(sm.W3);
  constexpr uint32_t idesc64 = tc05::idesc_bf16_f32<128, NH>(), idesc16 = tc05::idesc_bf16_f32<128, 16>();
  uint8_t *const xrow1 = sm.X + tc05::canon_off(t, 0, kSboA1);    // this thread's row of each A operand
  uint8_t *const xrow2 = sm.X + tc05::canon_off(t, 0, kSboA2);
  unsigned phase = 0;
  bool failed = false, bail = false;
  unsigned st = 0;
  const long ntiles = (n + TC_THREADS - 1) / TC_THREADS;
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long i = tile * TC_THREADS + t;
    const bool valid = i < n;
    Side L, R;
    Gas G;
    load_or_dummy(S, n, i, valid, L, R, G);
    const SideK kl = side_k(L, G), kr = side_k(R, G);
    const bool vac = vacuum(L, R, G);
    const double wtr = vac ? 0.0 : tr_w(L, R, kl, kr, G);
    const double ptr = vac ? 0.0 : p_of_w(wtr, G);
    const bool net = SOLVE ? (valid && !vac && !tr_exact(L, R, ptr) && strong_waves(L, R)) : (valid && !vac);
    float y = 0.f;
    {
      // layer-1 row: the features (zeros where the network is not
      // consulted), then the bias inputs
      float f[NIN];
      if (net) features(L, R, G.g, ptr, f);
      else for (int k = 0; k < NIN; ++k) f[k] = 0.f;
      *reinterpret_cast<uint4 *>(xrow1) =
          make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
      *reinterpret_cast<uint4 *>(xrow1 + kLbo) = ones;
    }
    tc05::fence_smem_to_async();
    tc05::fence_before_sync();
    const bool any = __syncthreads_or(net);
    if (sm.fail) { bail = true; break; }
    if (any) {
      if (t == 0) {
        tc05::fence_after_sync();
        tc05::mma_bf16(tmem, tc05::sdesc(xs, kLbo, kSboA1), tc05::sdesc(w1s, kLbo, kSboA1), idesc64, 0u);
        tc05::commit(&sm.bar);
      }
      failed |= !tc05::mbar_wait(&sm.bar, phase, kTcWaitCycles);
      phase ^= 1u;
      tc05::fence_after_sync();
      // hidden layer 1 (bias included) -> BF16 rows of layer 2, then its
      // bias inputs and padding
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t r[32];
        tc05::ld32(trow + half * 32, r);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4 *>(xrow2 + (half * 4 + q) * kLbo) = make_uint4(
              relu_bf16x2(__uint_as_float(r[8 * q + 0]), __uint_as_float(r[8 * q + 1])),
              relu_bf16x2(__uint_as_float(r[8 * q + 2]), __uint_as_float(r[8 * q + 3])),
              relu_bf16x2(__uint_as_float(r[8 * q + 4]), __uint_as_float(r[8 * q + 5])),
              relu_bf16x2(__uint_as_float(r[8 * q + 6]), __uint_as_float(r[8 * q + 7])));
      }
      *reinterpret_cast<uint4 *>(xrow2 + 8 * kLbo) = ones;
      *reinterpret_cast<uint4 *>(xrow2 + 9 * kLbo) = make_uint4(0u, 0u, 0u, 0u);
      tc05::fence_smem_to_async();
      tc05::fence_before_sync();
      if ((bail = __syncthreads_or(failed))) break;
      if (t == 0) {
        tc05::fence_after_sync();
#pragma unroll
        for (int kk = 0; kk < kK2 / 16; ++kk)
          tc05::mma_bf16(tmem, tc05::sdesc(xs + 256u * kk, kLbo, kSboA2), tc05::sdesc(w2s + 256u * kk, kLbo, kSboA2),
                         idesc64, kk > 0 ? 1u : 0u);
        tc05::commit(&sm.bar);
      }
      failed |= !tc05::mbar_wait(&sm.bar, phase, kTcWaitCycles);
      phase ^= 1u;
      tc05::fence_after_sync();
      // hidden layer 2 (bias included) -> BF16 rows of layer 3
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t r[32];
        tc05::ld32(trow + half * 32, r);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4 *>(xrow2 + (half * 4 + q) * kLbo) = make_uint4(
              relu_bf16x2(__uint_as_float(r[8 * q + 0]), __uint_as_float(r[8 * q + 1])),
              relu_bf16x2(__uint_as_float(r[8 * q + 2]), __uint_as_float(r[8 * q + 3])),
              relu_bf16x2(__uint_as_float(r[8 * q + 4]), __uint_as_float(r[8 * q + 5])),
              relu_bf16x2(__uint_as_float(r[8 * q + 6]), __uint_as_float(r[8 * q + 7])));
      }
      tc05::fence_smem_to_async();
      tc05::fence_before_sync();
      if ((bail = __syncthreads_or(failed))) break;
      if (t == 0) {
        tc05::fence_after_sync();
#pragma unroll
        for (int kk = 0; kk < NH / 16; ++kk)
          tc05::mma_bf16(tmem, tc05::sdesc(xs + 256u * kk, kLbo, kSboA2), tc05::sdesc(w3s + 256u * kk, kLbo, kSboW3),
                         idesc16, kk > 0 ? 1u : 0u);
        tc05::commit(&sm.bar);
      }
      if (!tc05::mbar_wait(&sm.bar, phase, kTcWaitCycles)) { failed = true; sm.fail = 1; }
      phase ^= 1u;
      tc05::fence_after_sync();
      uint32_t r2[2];
      tc05::ld2(trow, r2);
      y = (__uint_as_float(r2[0]) + __uint_as_float(r2[1])) + sm.b3;
      tc05::fence_before_sync();
    }
    if (SOLVE) {
      double w0 = wtr;
      if (net) w0 = wtr * (double)expf(float(G.z) * fminf(fmaxf(y, -20.f), 20.f));   // (p*/p_TR)^z
      const bool pending = solve_store(L, R, kl, kr, G, vac, net, w0, tol, max_iter, valid, i, n, out, iters,
                                       flags, st);
      enqueue(pending && valid, i, queue, qcount);
    } else if (valid) {
      yout[i] = net ? y : 0.f;
    }
  }
  if (!bail) bail = __syncthreads_or(sm.fail != 0);
  if (bail) {
    // the MMA of the phase that timed out may still be in flight
    if (t == 0) st |= FLASH_HY_ERR_TIMEOUT;
    if (failed) tc05::mbar_wait(&sm.bar, phase ^ 1u, kTcWaitCycles);
  }
  if (st) atomicOr(status, st);
  tc05::fence_before_sync();
  __syncthreads();
  if (wid == 0) {
    tc05::fence_after_sync();
    tc05::tmem_free(tmem, TC_TMEM_COLS);
  }
}

// fallback: queued solves restart from the two-rarefaction guess
__global__ void __launch_bounds__(SOLVE_THREADS) k_fallback(const double *__restrict__ S, long n,
                                                            double *__restrict__ out, unsigned char *__restrict__ iters,
                                                            unsigned char *__restrict__ flags, const int *queue,
                                                            const int *qcount, double tol, int max_iter,
                                                            unsigned *status) {
  const int nq = *qcount;
  unsigned st = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    const long i = queue[q];
    Side L, R;
    Gas G;
    load_state(S, n, i, L, R, G);
    Star S;
    unsigned char fl = 1 | 8;
    const SideK kl = side_k(L, G), kr = side_k(R, G);
    int k = newton(L, R, kl, kr, G, tr_w(L, R, kl, kr, G), tol, max_iter, S);
    int its = 3 + (k > 0 ? k : max_iter);
    if (k <= 0) { fl |= 4; st |= FLASH_HY_ERR_NEWTON_NOCONV; }
    out[i] = S.p; out[n + i] = S.u;
    if (iters) iters[i] = (unsigned char)(its > 255 ? 255 : its);
    if (flags) flags[i] = fl;
  }
  if (st) atomicOr(status, st);
}

// network output y = MLP(features) for every interface (0 for vacuum cases)
__global__ void __launch_bounds__(SOLVE_THREADS) k_predict(const double *__restrict__ S, long n, float *__restrict__ y,
                                                           const MlpPacked *__restrict__ w) {
  __shared__ __align__(16) MlpPacked M;
  load_packed(M, w);
  __syncthreads();
  for (long base = (long)blockIdx.x * blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
    const long i = base + threadIdx.x;
    float f[NIN];
    for (int k = 0; k < NIN; ++k) f[k] = 0.f;
    bool vac = true;
    if (i < n) {
      Side L, R;
      Gas G;
      load_state(S, n, i, L, R, G);
      vac = vacuum(L, R, G);
      if (!vac) features(L, R, G.g, tr_guess(L, R, G), f);
    }
    const float yy = mlp_lane(M, f);
    if (i < n) y[i] = vac ? 0.f : yy;
  }
}

// ---------------------------------------------------------------------------
// input generator of the isolated-solve workload (log-uniform pressure and
// density ratios over 1e8 and 1e6, velocities up to 5 sound speeds, gamma
// 7/5 or 5/3): splitmix64 of (seed, index, stream)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double uni(uint64_t seed, long i, int k) {
  uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)i * 8 + (uint64_t)k));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);     // [0, 1)
}

__global__ void k_generate(uint64_t seed, long n, double *S) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double g = uni(seed, i, 0) < 0.5 ? 1.4 : 5.0 / 3.0;
    double pr = exp(log(1e-4) + uni(seed, i, 1) * (log(1e4) - log(1e-4)));     // pR/pL log-uniform
    double dr = exp(log(1e-3) + uni(seed, i, 2) * (log(1e3) - log(1e-3)));     // rhoR/rhoL log-uniform
    double cl = sqrt(g), cr = sqrt(g * pr / dr);
    double ul = (2.0 * uni(seed, i, 3) - 1.0) * 5.0 * cl;
    double ur = (2.0 * uni(seed, i, 4) - 1.0) * 5.0 * cr;
    S[i] = 1.0; S[n + i] = ul; S[2 * n + i] = 1.0;
    S[3 * n + i] = dr; S[4 * n + i] = ur; S[5 * n + i] = pr; S[6 * n + i] = g;
  }
}

// ---------------------------------------------------------------------------
// training set: features and targets ln(p*/p_TR) of non-vacuum solves
// ---------------------------------------------------------------------------
__global__ void k_make_samples(const double *S, const double *out, long n, float *X, float *T, int *count, long cap) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    Side L, R;
    Gas G;
    load_state(S, n, i, L, R, G);
    if (vacuum(L, R, G)) continue;
    double ps = out[i];
    if (!(ps > 0.0)) continue;
    double ptr = tr_guess(L, R, G);
    if (tr_exact(L, R, ptr) || !strong_waves(L, R)) continue;   // where the network is consulted
    int k = atomicAdd(count, 1);
    if (k >= cap) continue;
    float f[NIN];
    features(L, R, G.g, ptr, f);
    for (int q = 0; q < NIN; ++q) X[(long)k * NIN + q] = f[q];
    T[k] = float(log(ps / ptr));
  }
}

// ---------------------------------------------------------------------------
// FP32 forward/backward of one minibatch (MSE, mean over the batch); each
// CTA handles TS samples and adds its gradient into G (atomics)
// ---------------------------------------------------------------------------
constexpr int TS = 32, TRAIN_THREADS = 256;

__global__ void __launch_bounds__(TRAIN_THREADS) k_grad(const float *__restrict__ w, const float *__restrict__ X,
                                                        const float *__restrict__ T, const int *__restrict__ idx, int nb,
                                                        float inv_batch, float *__restrict__ G, float *__restrict__ loss) {
  __shared__ float sW1[NH * NIN], sB1[NH], sW2[NH * NH], sB2[NH], sW3[NH];
  __shared__ float sX[TS][NIN], sH1[TS][NH + 1], sH2[TS][NH + 1], sD[TS];
  __shared__ float gW1[NH * NIN], gB1[NH], gW3[NH], gB2[NH];
  const int tid = threadIdx.x;
  for (int t = tid; t < NH * NIN; t += TRAIN_THREADS) { sW1[t] = w[OFF_W1 + t]; gW1[t] = 0.f; }
  for (int t = tid; t < NH * NH; t += TRAIN_THREADS) sW2[t] = w[OFF_W2 + t];
  for (int t = tid; t < NH; t += TRAIN_THREADS) {
    sB1[t] = w[OFF_B1 + t]; sB2[t] = w[OFF_B2 + t]; sW3[t] = w[OFF_W3 + t];
    gB1[t] = 0.f; gW3[t] = 0.f; gB2[t] = 0.f;
  }
  const float b3 = w[OFF_B3];
  const int s0 = blockIdx.x * TS;
  const int ns = min(TS, nb - s0);
  for (int t = tid; t < TS * NIN; t += TRAIN_THREADS) {
    int s = t / NIN, k = t % NIN;
    sX[s][k] = s < ns ? X[(long)idx[s0 + s] * NIN + k] : 0.f;
  }
  __syncthreads();
  // forward
  for (int t = tid; t < TS * NH; t += TRAIN_THREADS) {
    int s = t / NH, u = t % NH;
    float a = sB1[u];
#pragma unroll
    for (int k = 0; k < NIN; ++k) a += sW1[u * NIN + k] * sX[s][k];
    sH1[s][u] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int t = tid; t < TS * NH; t += TRAIN_THREADS) {
    int s = t / NH, u = t % NH;
    float a = sB2[u];
    for (int j = 0; j < NH; ++j) a += sW2[u * NH + j] * sH1[s][j];
    sH2[s][u] = fmaxf(a, 0.f);
  }
  __syncthreads();
  // output and dL/dy per sample (one warp per group of samples)
  float lsum = 0.f;
  for (int s = tid >> 5; s < TS; s += TRAIN_THREADS / 32) {
    float a = 0.f;
    for (int u = tid & 31; u < NH; u += 32) a += sW3[u] * sH2[s][u];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((tid & 31) == 0) {
      float y = a + b3;
      float r = s < ns ? y - T[idx[s0 + s]] : 0.f;
      sD[s] = 2.f * r * inv_batch;
      lsum += r * r;
    }
  }
  __syncthreads();
  // dH2 (in place over sH2 after using it for dW3)
  for (int u = tid; u < NH; u += TRAIN_THREADS) {
    float gw = 0.f;
    for (int s = 0; s < TS; ++s) gw += sD[s] * sH2[s][u];
    gW3[u] = gw;
  }
  __syncthreads();
  for (int t = tid; t < TS * NH; t += TRAIN_THREADS) {
    int s = t / NH, u = t % NH;
    sH2[s][u] = sH2[s][u] > 0.f ? sD[s] * sW3[u] : 0.f;
  }
  __syncthreads();
  // dW2[u][j] = sum_s dH2[s][u] H1[s][j], db2
  for (int t = tid; t < NH * NH; t += TRAIN_THREADS) {
    int u = t / NH, j = t % NH;
    float a = 0.f;
    for (int s = 0; s < TS; ++s) a += sH2[s][u] * sH1[s][j];
    atomicAdd(&G[OFF_W2 + t], a);
  }
  for (int u = tid; u < NH; u += TRAIN_THREADS) {
    float a = 0.f;
    for (int s = 0; s < TS; ++s) a += sH2[s][u];
    gB2[u] = a;
  }
  // dH1 = (dH2 W2) relu'(H1), written into a register pass then sH1
  __syncthreads();
  float dh1[TS * NH / TRAIN_THREADS];
#pragma unroll
  for (int q = 0; q < TS * NH / TRAIN_THREADS; ++q) {
    int t = tid + q * TRAIN_THREADS;
    int s = t / NH, j = t % NH;
    float a = 0.f;
    for (int u = 0; u < NH; ++u) a += sH2[s][u] * sW2[u * NH + j];
    dh1[q] = sH1[s][j] > 0.f ? a : 0.f;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < TS * NH / TRAIN_THREADS; ++q) {
    int t = tid + q * TRAIN_THREADS;
    sH1[t / NH][t % NH] = dh1[q];
  }
  __syncthreads();
  for (int t = tid; t < NH * NIN; t += TRAIN_THREADS) {
    int j = t / NIN, k = t % NIN;
    float a = 0.f;
    for (int s = 0; s < TS; ++s) a += sH1[s][j] * sX[s][k];
    gW1[t] = a;
  }
  for (int j = tid; j < NH; j += TRAIN_THREADS) {
    float a = 0.f;
    for (int s = 0; s < TS; ++s) a += sH1[s][j];
    gB1[j] = a;
  }
  __syncthreads();
  for (int t = tid; t < NH * NIN; t += TRAIN_THREADS) atomicAdd(&G[OFF_W1 + t], gW1[t]);
  for (int t = tid; t < NH; t += TRAIN_THREADS) {
    atomicAdd(&G[OFF_B1 + t], gB1[t]);
    atomicAdd(&G[OFF_B2 + t], gB2[t]);
    atomicAdd(&G[OFF_W3 + t], gW3[t]);
  }
  if (tid == 0) {
    float a = 0.f;
    for (int s = 0; s < TS; ++s) a += sD[s];
    atomicAdd(&G[OFF_B3], a);
  }
  // loss (sum of squared residuals of this CTA)
  if ((tid & 31) == 0) atomicAdd(loss, lsum);
}

__global__ void k_adam(float *w, float *m, float *v, const float *G, int step, float lr, float b1, float b2, float eps) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NPARAM) return;
  float g = G[t];
  m[t] = b1 * m[t] + (1.f - b1) * g;
  v[t] = b2 * v[t] + (1.f - b2) * g * g;
  float mh = m[t] / (1.f - powf(b1, (float)step));
  float vh = v[t] / (1.f - powf(b2, (float)step));
  w[t] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_shuffle_idx(int *idx, int n, uint64_t seed) {
  // one random key per sample, then the host sorts nothing: a multiplicative
  // permutation (a*i + c) mod n with a coprime to n visits every sample once
  long a = 1 + 2 * (long)(splitmix64(seed) % (uint64_t)(n > 2 ? n / 2 : 1));
  while (true) {
    long x = a, y = n, t;
    while (y) { t = x % y; x = y; y = t; }
    if (x == 1) break;
    a += 2;
  }
  long c = (long)(splitmix64(seed + 1) % (uint64_t)n);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    idx[i] = (int)((a * i + c) % n);
}

}  // namespace rx

using namespace rx;

struct flash_hy_rsolver {
  int device;
  cudaStream_t stream;
  float *w, *m, *v, *G, *loss;
  MlpPacked *packed;            // BF16 inference copy of w
  int *queue, *qcount;          // fallback queue of the learned path
  long qcap;
  unsigned *status;
  int step;
  int infer;                    // FLASH_HY_INFER_TCGEN05 or FLASH_HY_INFER_WARP_MMA
  int tc_grid, tc_grid_p;       // resident CTAs of k_solve_tc<true> / <false> over the device
  char err[256];
};

#define RS_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) { snprintf(r->err, sizeof r->err, "CUDA: %s", cudaGetErrorString(e_)); return FLASH_HY_ERR_CUDA; } \
  } while (0)

static int grid_for(long n, int threads) {
  long g = (n + threads - 1) / threads;
  if (g > 148L * 16) g = 148L * 16;
  return (int)(g > 0 ? g : 1);
}

static int repack(flash_hy_rsolver *r) {
  k_pack_mlp<<<1, 256, 0, r->stream>>>(r->w, r->packed);
  RS_CUDA(cudaGetLastError());
  return 0;
}

// CTAs of a tcgen05 kernel that fit on one SM at once, from its registers
// (allocated per warp in units of 256), its shared memory (plus the 1 KB the
// driver reserves per CTA), the SM's 64 warps and its 512 TMEM columns
// (TC_TMEM_COLS per CTA); the grids below launch that many per SM, so no
// CTA waits in tcgen05.alloc.  (The runtime's occupancy query answers 1 for
// these kernels.)
static int tc_ctas_per_sm(const void *kernel, int device, int &out) {
  cudaFuncAttributes fa;
  int regs_sm = 0, smem_sm = 0, warps_sm = 0;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&warps_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device) != cudaSuccess)
    return FLASH_HY_ERR_CUDA;
  const int warps = TC_THREADS / 32;
  const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
  int n = regs_sm / (regs_warp * warps);
  const int by_smem = smem_sm / ((int)fa.sharedSizeBytes + 1024);
  const int by_warps = warps_sm / 32 / warps;
  const int by_tmem = 512 / (int)TC_TMEM_COLS;
  if (by_smem < n) n = by_smem;
  if (by_warps < n) n = by_warps;
  if (by_tmem < n) n = by_tmem;
  out = n > 0 ? n : 1;
  return 0;
}

extern "C" int flash_hy_rsolver_create(int device, flash_hy_rsolver **out) {
  if (!out) return FLASH_HY_ERR_BAD_ARG;
  flash_hy_rsolver *r = (flash_hy_rsolver *)calloc(1, sizeof *r);
  *out = r;
  r->device = device;
  RS_CUDA(cudaSetDevice(device));
  RS_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
  RS_CUDA(cudaMalloc(&r->w, NPARAM * sizeof(float)));
  RS_CUDA(cudaMalloc(&r->m, NPARAM * sizeof(float)));
  RS_CUDA(cudaMalloc(&r->v, NPARAM * sizeof(float)));
  RS_CUDA(cudaMalloc(&r->G, NPARAM * sizeof(float)));
  RS_CUDA(cudaMalloc(&r->loss, sizeof(float)));
  RS_CUDA(cudaMalloc(&r->status, sizeof(unsigned)));
  RS_CUDA(cudaMalloc(&r->qcount, sizeof(int)));
  RS_CUDA(cudaMalloc(&r->packed, sizeof(MlpPacked)));
  RS_CUDA(cudaMemset(r->m, 0, NPARAM * sizeof(float)));
  RS_CUDA(cudaMemset(r->v, 0, NPARAM * sizeof(float)));
  RS_CUDA(cudaMemset(r->status, 0, sizeof(unsigned)));
  // He-style initialisation from a fixed seed (host side, deterministic)
  float *h = (float *)malloc(NPARAM * sizeof(float));
  uint64_t s = 12345;
  auto rnd = [&]() { s = s * 6364136223846793005ull + 1442695040888963407ull; return ((s >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0; };
  for (int t = 0; t < NPARAM; ++t) h[t] = 0.f;
  for (int t = 0; t < NH * NIN; ++t) h[OFF_W1 + t] = (float)(rnd() * sqrt(6.0 / NIN));
  for (int t = 0; t < NH * NH; ++t) h[OFF_W2 + t] = (float)(rnd() * sqrt(6.0 / NH));
  for (int t = 0; t < NH; ++t) h[OFF_W3 + t] = (float)(rnd() * sqrt(3.0 / NH) * 0.1);
  cudaError_t e = cudaMemcpy(r->w, h, NPARAM * sizeof(float), cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess) return FLASH_HY_ERR_CUDA;
  int sms = 0;
  RS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  int occ_s = 0, occ_p = 0;
  if (int e2 = tc_ctas_per_sm((const void *)k_solve_tc<true>, device, occ_s)) return e2;
  if (int e2 = tc_ctas_per_sm((const void *)k_solve_tc<false>, device, occ_p)) return e2;
  r->tc_grid = sms * occ_s;
  r->tc_grid_p = sms * occ_p;
  r->infer = FLASH_HY_INFER_TCGEN05;
  return repack(r);
}

extern "C" int flash_hy_rsolver_set_inference(flash_hy_rsolver *r, int mode) {
  if (!r || (mode != FLASH_HY_INFER_TCGEN05 && mode != FLASH_HY_INFER_WARP_MMA)) return FLASH_HY_ERR_BAD_ARG;
  r->infer = mode;
  return 0;
}

static int tc_grid_for(long n, int resident) {
  const long tiles = (n + TC_THREADS - 1) / TC_THREADS;
  return (int)(tiles < resident ? tiles : resident);
}

extern "C" int flash_hy_rsolver_destroy(flash_hy_rsolver *r) {
  if (!r) return FLASH_HY_ERR_BAD_ARG;
  cudaSetDevice(r->device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  cudaFree(r->w); cudaFree(r->m); cudaFree(r->v); cudaFree(r->G); cudaFree(r->loss); cudaFree(r->status);
  cudaFree(r->queue); cudaFree(r->qcount); cudaFree(r->packed);
  if (r->stream) cudaStreamDestroy(r->stream);
  free(r);
  return 0;
}

extern "C" void *flash_hy_rsolver_stream(flash_hy_rsolver *r) { return r ? (void *)r->stream : nullptr; }

extern "C" int flash_hy_rsolver_generate(flash_hy_rsolver *r, unsigned long long seed, long n, double *d_states) {
  if (!r || !d_states || n <= 0) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  k_generate<<<grid_for(n, 256), 256, 0, r->stream>>>(seed, n, d_states);
  RS_CUDA(cudaGetLastError());
  return 0;
}

extern "C" int flash_hy_rsolver_solve(flash_hy_rsolver *r, const double *d_states, long n, double *d_star,
                                      unsigned char *d_iters, unsigned char *d_flags, int learned, double tol,
                                      int max_iter) {
  if (!r || !d_states || !d_star || n <= 0 || n > 0x7fffffffL || max_iter <= 0 || max_iter > 200)
    return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  if (learned && r->qcap < n) {
    if (r->queue) { cudaStreamSynchronize(r->stream); cudaFree(r->queue); r->queue = nullptr; r->qcap = 0; }
    RS_CUDA(cudaMalloc(&r->queue, n * sizeof(int)));
    r->qcap = n;
  }
  if (learned) RS_CUDA(cudaMemsetAsync(r->qcount, 0, sizeof(int), r->stream));
  if (learned && r->infer == FLASH_HY_INFER_TCGEN05)
    k_solve_tc<true><<<tc_grid_for(n, r->tc_grid), TC_THREADS, 0, r->stream>>>(
        d_states, n, d_star, d_iters, d_flags, r->packed, tol, max_iter, r->queue, r->qcount, r->status, nullptr);
  else if (learned)
    k_solve<true><<<grid_for(n, SOLVE_THREADS), SOLVE_THREADS, 0, r->stream>>>(
        d_states, n, d_star, d_iters, d_flags, r->packed, tol, max_iter, r->queue, r->qcount, r->status);
  else
    k_solve<false><<<grid_for(n, SOLVE_THREADS), SOLVE_THREADS, 0, r->stream>>>(
        d_states, n, d_star, d_iters, d_flags, r->packed, tol, max_iter, r->queue, r->qcount, r->status);
  RS_CUDA(cudaGetLastError());
  if (learned) {
    k_fallback<<<148 * 4, SOLVE_THREADS, 0, r->stream>>>(d_states, n, d_star, d_iters, d_flags, r->queue, r->qcount,
                                                         tol, max_iter, r->status);
    RS_CUDA(cudaGetLastError());
  }
  return 0;
}

extern "C" int flash_hy_rsolver_predict(flash_hy_rsolver *r, const double *d_states, long n, float *d_y) {
  if (!r || !d_states || !d_y || n <= 0) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  if (r->infer == FLASH_HY_INFER_TCGEN05)
    k_solve_tc<false><<<tc_grid_for(n, r->tc_grid_p), TC_THREADS, 0, r->stream>>>(
        d_states, n, nullptr, nullptr, nullptr, r->packed, 0.0, 0, nullptr, nullptr, r->status, d_y);
  else
    k_predict<<<grid_for(n, SOLVE_THREADS), SOLVE_THREADS, 0, r->stream>>>(d_states, n, d_y, r->packed);
  RS_CUDA(cudaGetLastError());
  return 0;
}

extern "C" int flash_hy_rsolver_make_samples(flash_hy_rsolver *r, const double *d_states, const double *d_star, long n,
                                             float *d_x, float *d_t, long cap, long *count_out) {
  if (!r || !d_states || !d_star || !d_x || !d_t || !count_out) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  int *cnt;
  RS_CUDA(cudaMalloc(&cnt, sizeof(int)));
  RS_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), r->stream));
  k_make_samples<<<grid_for(n, 256), 256, 0, r->stream>>>(d_states, d_star, n, d_x, d_t, cnt, cap);
  int h = 0;
  RS_CUDA(cudaMemcpyAsync(&h, cnt, sizeof(int), cudaMemcpyDeviceToHost, r->stream));
  RS_CUDA(cudaStreamSynchronize(r->stream));
  cudaFree(cnt);
  *count_out = h < cap ? h : cap;
  return 0;
}

// Gradient of the mean-squared loss on samples idx[0..nb) (device arrays);
// writes the FP32 gradient (NPARAM floats) and the loss to host memory.
extern "C" int flash_hy_rsolver_grad(flash_hy_rsolver *r, const float *d_x, const float *d_t, const int *d_idx, int nb,
                                     float *h_grad, float *h_loss) {
  if (!r || !d_x || !d_t || !d_idx || nb <= 0) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  RS_CUDA(cudaMemsetAsync(r->G, 0, NPARAM * sizeof(float), r->stream));
  RS_CUDA(cudaMemsetAsync(r->loss, 0, sizeof(float), r->stream));
  k_grad<<<(nb + TS - 1) / TS, TRAIN_THREADS, 0, r->stream>>>(r->w, d_x, d_t, d_idx, nb, 1.f / nb, r->G, r->loss);
  RS_CUDA(cudaGetLastError());
  if (h_grad) RS_CUDA(cudaMemcpyAsync(h_grad, r->G, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
  if (h_loss) RS_CUDA(cudaMemcpyAsync(h_loss, r->loss, sizeof(float), cudaMemcpyDeviceToHost, r->stream));
  RS_CUDA(cudaStreamSynchronize(r->stream));
  if (h_loss) *h_loss /= nb;
  return 0;
}

// Adam training over ns samples (device arrays from make_samples): epochs x
// minibatches of `batch`; returns the mean loss of the last epoch.
extern "C" int flash_hy_rsolver_train(flash_hy_rsolver *r, const float *d_x, const float *d_t, long ns, int epochs,
                                      int batch, float lr, float *loss_out) {
  if (!r || !d_x || !d_t || ns < batch || batch <= 0 || epochs <= 0) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  int *idx;
  RS_CUDA(cudaMalloc(&idx, ns * sizeof(int)));
  float last = 0.f;
  long nbat = ns / batch;
  for (int ep = 0; ep < epochs; ++ep) {
    k_shuffle_idx<<<grid_for(ns, 256), 256, 0, r->stream>>>(idx, (int)ns, 0x5eedull + ep);
    RS_CUDA(cudaMemsetAsync(r->loss, 0, sizeof(float), r->stream));
    for (long bi = 0; bi < nbat; ++bi) {
      RS_CUDA(cudaMemsetAsync(r->G, 0, NPARAM * sizeof(float), r->stream));
      k_grad<<<(batch + TS - 1) / TS, TRAIN_THREADS, 0, r->stream>>>(r->w, d_x, d_t, idx + bi * batch, batch,
                                                                      1.f / batch, r->G, r->loss);
      r->step++;
      float lr_ep = lr * powf(0.05f, (float)ep / (float)epochs);   // exponential decay to lr/20
      k_adam<<<(NPARAM + 255) / 256, 256, 0, r->stream>>>(r->w, r->m, r->v, r->G, r->step, lr_ep, 0.9f, 0.999f, 1e-8f);
    }
    float h = 0.f;
    RS_CUDA(cudaMemcpyAsync(&h, r->loss, sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    RS_CUDA(cudaStreamSynchronize(r->stream));
    last = h / (float)(nbat * batch);
  }
  cudaFree(idx);
  RS_CUDA(cudaGetLastError());
  if (loss_out) *loss_out = last;
  return repack(r);
}

extern "C" int flash_hy_rsolver_get_weights(flash_hy_rsolver *r, float *h_w, int n) {
  if (!r || !h_w || n < NPARAM) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  RS_CUDA(cudaMemcpy(h_w, r->w, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int flash_hy_rsolver_set_weights(flash_hy_rsolver *r, const float *h_w, int n) {
  if (!r || !h_w || n < NPARAM) return FLASH_HY_ERR_BAD_ARG;
  RS_CUDA(cudaSetDevice(r->device));
  RS_CUDA(cudaMemcpy(r->w, h_w, NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemset(r->m, 0, NPARAM * sizeof(float)));
  RS_CUDA(cudaMemset(r->v, 0, NPARAM * sizeof(float)));
  r->step = 0;
  return repack(r);
}

extern "C" int flash_hy_rsolver_num_params(void) { return NPARAM; }

extern "C" int flash_hy_rsolver_sync(flash_hy_rsolver *r) {
  if (!r) return FLASH_HY_ERR_BAD_ARG;
  unsigned h = 0;
  RS_CUDA(cudaSetDevice(r->device));
  RS_CUDA(cudaMemcpyAsync(&h, r->status, sizeof(unsigned), cudaMemcpyDeviceToHost, r->stream));
  RS_CUDA(cudaMemsetAsync(r->status, 0, sizeof(unsigned), r->stream));
  RS_CUDA(cudaStreamSynchronize(r->stream));
  return (int)h;
}
