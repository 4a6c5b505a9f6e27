// mpnn.cu -- learned JCG initial guess: a message-passing network over each
// node's 1-ring, with BF16 tensor-core (mma.sync m16n8k16, FP32 accumulate)
// kernels for inference and for training on the device.
//
// The reference starts JCG from ETAS as GWCE_New leaves it (gwce.F:
// 1846-1850, 2002-2004: the previous increment at interior nodes, the new
// boundary increment at elevation-specified nodes).  Here a network
// predicts a correction to that guess at wet interior nodes:
//
//   x_i   = normalised (eta^k, ETAS_ref, u, v, depth, wet flag, p - p_bg,
//           tau_x, tau_y) of node i, as BF16, plus a constant 1 (the bias)
//   h0_i  = ReLU(W_in x_i)                                   9+1 -> 64
//   h_l,i = ReLU(Ws_l h_l-1,i + Wn_l mean_{j in N(i)} h_l-1,j + b_l)   l = 1..3
//   ETAS_guess_i = ETAS_ref_i + s_out (w_out . h3_i + b_out)
//
// with s_out a fixed scale of the corrections (set with the weights).
// N(i) is the node's NeiTab ring (the GWCE matrix pattern).  Weights are
// FP32 masters with BF16 copies for the tensor-core passes; activations
// are stored in BF16, gradients in FP32.  JCG iterates to the unchanged
// tolerance from whichever of the two guesses has the smaller initial
// residual (warm.cu), so the network can cost iterations but not accuracy.
//
// Training (adc_predictor_train) runs after each step's solve on the pair
// (features before the solve, solved ETAS): Huber loss (quadratic within
// kHuber, linear beyond) of the normalised correction over wet interior
// nodes, so the few nodes at a moving wet/dry front do not dominate it; exact backpropagation through the
// head, the three message-passing layers and the input layer, weight
// gradients as per-CTA partial GEMMs summed in a fixed order, and an Adam
// update of the FP32 masters.  With ADC_LEARNED_START off the solver keeps
// the reference guess, so the training pairs are those of the plain solver.
#include "adc_internal.cuh"

#include <cstring>
#include <vector>

namespace adc {

constexpr int kF = 16;              // padded input width (9 features, 1 bias, 6 zero)
constexpr int kNF = 9;              // features
constexpr int kH = 64;              // hidden width
constexpr int kL = 3;               // message-passing layers
constexpr int kTile = 64;           // nodes per CTA tile
constexpr int kMpThreads = 128;     // 4 warps, 16 nodes each
constexpr float kHuber = 3.f;       // Huber threshold of the normalised error
constexpr int kNStats = 2;          // Mpnn::stats entries

// Flat FP32 parameter layout (adc_set_predictor / adc_get_predictor).
constexpr int kOffWin = 0;                                  // W_in [64][16]
constexpr int kOffLayer = kOffWin + kH * kF;                // per layer: Ws, Wn [64][64], b [64]
constexpr int kLayerSz = 2 * kH * kH + kH;
constexpr int kOffWout = kOffLayer + kL * kLayerSz;         // w_out [64]
constexpr int kOffBout = kOffWout + kH;                     // b_out
constexpr int kNTrain = kOffBout + 1;                       // trained parameters
constexpr int kOffNorm = kNTrain;                           // mean[9], std[9], s_out
constexpr int kNParams = kOffNorm + 2 * kNF + 1;

struct Mpnn {
  int n;                          // nodes
  float *par, *grad, *m1, *m2;    // FP32 masters, gradient, Adam moments (kNParams)
  __nv_bfloat16 *wbf;             // BF16 copies: W_in, then per layer [Ws | Wn] rows of 128
  __nv_bfloat16 *x;               // [n][16]
  __nv_bfloat16 *h[kL + 1];       // [n][64]
  __nv_bfloat16 *mean[kL];        // ring means of h[0..kL-1], [n][64]
  __nv_bfloat16 *adz;             // backward messages, [n][64]
  float *dz[2];                   // [n][64]
  double *ref;                    // ETAS_ref, [n]
  double *pred;                   // ETAS guess, [n]
  float *dout;                    // dL/d out, [n]
  int *nb_ptr, *nb_idx;           // 1-ring without the node itself
  float *inv_deg;                 // 1 / |N(i)|
  float *part;                    // per-CTA weight-gradient partials
  int part_ctas;
  int dense_ctas[3];              // persistent grid of k_mp_dense<0/1/2>
  double *loss_part;              // per-block loss partials
  double *stats;                  // [0] loss of the last step, [1] Adam steps
  const double *tgt;              // training target (the solved ETAS when null)
  int train, learned;
  float lr;
};

// ------------------------------------------------------------- mma helpers
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], unsigned a0, unsigned a1, unsigned a2,
                                         unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One warp: C[16 x 64] += A[16 x K] * B[K x 64], A row-major in shared
// memory (row stride sa, in BF16 elements), B given as its transpose
// Bt[64 x K] (row stride sb).  acc[nt][*] holds the C fragment of the 8
// column tiles nt (rows g and g+8, columns 8 nt + 2 t, +1).
template <int K>
__device__ __forceinline__ void warp_gemm_16x64(const __nv_bfloat16 *A, int sa,
                                                const __nv_bfloat16 *Bt, int sb,
                                                float (&acc)[8][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    const unsigned a0 = *reinterpret_cast<const unsigned *>(A + g * sa + k0 + 2 * t);
    const unsigned a1 = *reinterpret_cast<const unsigned *>(A + (g + 8) * sa + k0 + 2 * t);
    const unsigned a2 = *reinterpret_cast<const unsigned *>(A + g * sa + k0 + 2 * t + 8);
    const unsigned a3 = *reinterpret_cast<const unsigned *>(A + (g + 8) * sa + k0 + 2 * t + 8);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __nv_bfloat16 *b = Bt + (nt * 8 + g) * sb + k0 + 2 * t;
      mma_bf16(acc[nt], a0, a1, a2, a3, *reinterpret_cast<const unsigned *>(b),
               *reinterpret_cast<const unsigned *>(b + 8));
    }
  }
}

struct MpArgs {
  int n;
  const __nv_bfloat16 *wbf;
  const float *par;
  const int *nb_ptr, *nb_idx;
  const float *inv_deg;
};

// Shared-memory row strides (BF16 elements), padded against bank conflicts.
constexpr int kSA = 2 * kH + 8;     // A rows of up to 128
constexpr int kSX = kF + 8;

// Neighbour gathers.  A tile's 64 nodes have contiguous CSR slices, so a
// CTA stages the tile's ring pointers and (when they fit) its neighbour
// indices in shared memory with coalesced loads; then 8 lanes share a node,
// each summing 8 channels of the neighbours' rows with 16-byte loads, the
// first kRing neighbours' rows requested together.  Every channel sums its
// neighbours in NeiTab order.
constexpr int kIdxCap = 1024;       // staged neighbour indices per tile
constexpr int kRing = 8;            // neighbour rows requested together

template <bool W>
struct TileRing {
  int ptr[kTile + 1];
  int idx[kIdxCap];
  float w[W ? kIdxCap : 1];         // 1/deg of each neighbour (dz sums)
};

// Stages the CSR slice of the tile at node0; returns whether its indices
// fit in shared memory (otherwise they are read from global memory).
template <bool W>
__device__ bool stage_ring(const MpArgs &a, int node0, TileRing<W> &s) {
  const int nt = min(kTile, a.n - node0);
  for (int t = threadIdx.x; t <= nt; t += blockDim.x) s.ptr[t] = a.nb_ptr[node0 + t];
  __syncthreads();
  const int base = s.ptr[0], cnt = s.ptr[nt] - base;
  const bool fit = cnt <= kIdxCap;
  if (fit)
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      const int j = a.nb_idx[base + q];
      s.idx[q] = j;
      if (W) s.w[q] = a.inv_deg[j];
    }
  __syncthreads();
  return fit;
}

__device__ __forceinline__ void add_bf16x8(float (&acc)[8], const uint4 &v) {
  const __nv_bfloat162 *b = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float2 f = __bfloat1622float2(b[e]);
    acc[2 * e] += f.x;
    acc[2 * e + 1] += f.y;
  }
}

__device__ __forceinline__ void unpack_bf16x8(float (&o)[8], const uint4 &v) {
  const __nv_bfloat162 *b = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float2 f = __bfloat1622float2(b[e]);
    o[2 * e] = f.x;
    o[2 * e + 1] = f.y;
  }
}

__device__ __forceinline__ uint4 pack_bf16x8(const float (&v)[8]) {
  uint4 o;
  o.x = pack_bf16(v[0], v[1]);
  o.y = pack_bf16(v[2], v[3]);
  o.z = pack_bf16(v[4], v[5]);
  o.w = pack_bf16(v[6], v[7]);
  return o;
}

// Row r of the staged tile: sum over its ring of h_j[8 ch .. 8 ch + 7].
template <bool W>
__device__ __forceinline__ void ring_chunk_h(const MpArgs &a, const TileRing<W> &s, bool fit,
                                             const __nv_bfloat16 *h, int r, int ch, float (&acc)[8]) {
  const int p0 = s.ptr[r], deg = s.ptr[r + 1] - p0, o = p0 - s.ptr[0];
#pragma unroll
  for (int e = 0; e < 8; ++e) acc[e] = 0.f;
  for (int q0 = 0; q0 < deg; q0 += kRing) {
    uint4 v[kRing];
#pragma unroll
    for (int q = 0; q < kRing; ++q) {
      v[q] = make_uint4(0u, 0u, 0u, 0u);
      if (q0 + q < deg) {
        const int j = fit ? s.idx[o + q0 + q] : a.nb_idx[p0 + q0 + q];
        v[q] = reinterpret_cast<const uint4 *>(h + (size_t)j * kH)[ch];
      }
    }
#pragma unroll
    for (int q = 0; q < kRing; ++q)
      if (q0 + q < deg) add_bf16x8(acc, v[q]);
  }
}

// Row r of the staged tile: sum over its ring of dz_j[8 ch .. +7] / deg_j.
__device__ __forceinline__ void ring_chunk_dz(const MpArgs &a, const TileRing<true> &s, bool fit,
                                              const float *dz, int r, int ch, float (&acc)[8]) {
  const int p0 = s.ptr[r], deg = s.ptr[r + 1] - p0, o = p0 - s.ptr[0];
#pragma unroll
  for (int e = 0; e < 8; ++e) acc[e] = 0.f;
  for (int q0 = 0; q0 < deg; q0 += kRing / 2) {
    float4 v[kRing / 2][2];
    float w[kRing / 2];
#pragma unroll
    for (int q = 0; q < kRing / 2; ++q) {
      v[q][0] = v[q][1] = make_float4(0.f, 0.f, 0.f, 0.f);
      w[q] = 0.f;
      if (q0 + q < deg) {
        const int j = fit ? s.idx[o + q0 + q] : a.nb_idx[p0 + q0 + q];
        w[q] = fit ? s.w[o + q0 + q] : a.inv_deg[j];
        const float4 *row = reinterpret_cast<const float4 *>(dz + (size_t)j * kH) + 2 * ch;
        v[q][0] = row[0];
        v[q][1] = row[1];
      }
    }
#pragma unroll
    for (int q = 0; q < kRing / 2; ++q)
      if (q0 + q < deg) {
        acc[0] += v[q][0].x * w[q];
        acc[1] += v[q][0].y * w[q];
        acc[2] += v[q][0].z * w[q];
        acc[3] += v[q][0].w * w[q];
        acc[4] += v[q][1].x * w[q];
        acc[5] += v[q][1].y * w[q];
        acc[6] += v[q][1].z * w[q];
        acc[7] += v[q][1].w * w[q];
      }
  }
}

// ----------------------------------------------------------- the features
__global__ void k_mp_features(adc_ctx c, Mpnn m) {
  griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n) return;
  const float *mean = m.par + kOffNorm, *sd = mean + kNF;
  const double pb = c.p.prbckgrnd_mh2o;
  const double ref = c.etas[i];
  float f[kNF] = {(float)c.eta1[i],
                  (float)ref,
                  (float)c.uu1[i],
                  (float)c.vv1[i],
                  (float)c.dp[i],
                  (float)c.nodecode[i],
                  (float)(c.pr2[i] - pb),
                  (float)c.wsx2[i],
                  (float)c.wsy2[i]};
  __nv_bfloat16 *xo = m.x + (size_t)i * kF;
#pragma unroll
  for (int k = 0; k < kF; k += 2) {
    float lo = 0.f, hi = 0.f;
    if (k < kNF) lo = (f[k] - mean[k]) / sd[k];
    if (k + 1 < kNF) hi = (f[k + 1] - mean[k + 1]) / sd[k + 1];
    if (k + 1 == kNF) hi = 1.f;     // the bias input x[9], in the pair (8, 9)
    *reinterpret_cast<__nv_bfloat162 *>(xo + k) = __floats2bfloat162_rn(lo, hi);
  }
  m.ref[i] = ref;
}

// ------------------------------------------------------ ring aggregation
// The messages of one tile of 64 nodes per CTA (8 lanes per node):
// mean_i = BF16((1/|N(i)|) sum_{j in N(i)} h_j).
__global__ void __launch_bounds__(kMpThreads, 8) k_mp_aggr(MpArgs a, const __nv_bfloat16 *h,
                                                         __nv_bfloat16 *mean) {
  griddep_wait();
  __shared__ TileRing<false> ring;
  const int node0 = blockIdx.x * kTile;
  const bool fit = stage_ring<false>(a, node0, ring);
  const int ch = threadIdx.x & 7;
  for (int row = threadIdx.x >> 3; row < kTile; row += kMpThreads / 8) {
    const int i = node0 + row;
    if (i >= a.n) break;
    float agg[8];
    ring_chunk_h(a, ring, fit, h, row, ch, agg);
    const float sc = a.inv_deg[i];
#pragma unroll
    for (int e = 0; e < 8; ++e) agg[e] *= sc;
    reinterpret_cast<uint4 *>(mean + (size_t)i * kH)[ch] = pack_bf16x8(agg);
  }
}

// The backward messages: adz_i = BF16(sum_{j in N(i)} dz_j / |N(j)|).
__global__ void __launch_bounds__(kMpThreads, 8) k_mp_aggr_dz(MpArgs a, const float *dz,
                                                            __nv_bfloat16 *adz) {
  griddep_wait();
  __shared__ TileRing<true> ring;
  const int node0 = blockIdx.x * kTile;
  const bool fit = stage_ring<true>(a, node0, ring);
  const int ch = threadIdx.x & 7;
  for (int row = threadIdx.x >> 3; row < kTile; row += kMpThreads / 8) {
    const int i = node0 + row;
    if (i >= a.n) break;
    float agg[8];
    ring_chunk_dz(a, ring, fit, dz, row, ch, agg);
    reinterpret_cast<uint4 *>(adz + (size_t)i * kH)[ch] = pack_bf16x8(agg);
  }
}

// ----------------------------------------------------------- dense passes
// mode 0: h0 = ReLU(W_in x)                                  (K = 16)
// mode 1: h_l = ReLU([h_l-1 | mean_l-1] [Ws; Wn]^T + b)        (K = 128)
// mode 2: dz_l-1 = ([dz_l | adz_l] [Ws; Wn]) * (h_l-1 > 0)
// Persistent CTAs over tiles of 64 nodes: the weights are staged once per
// CTA; each thread loads its share of the next tile's rows into registers
// while the current tile's GEMM and store run.  Mode 0 and 1 stage the
// output tile in shared memory and write whole rows.
template <int MODE>
__global__ void __launch_bounds__(kMpThreads) k_mp_dense(MpArgs a, int layer,
                                                          const __nv_bfloat16 *hin,
                                                          const __nv_bfloat16 *msg,
                                                          const float *dzin,
                                                          __nv_bfloat16 *hout, float *dzout,
                                                          int ntiles) {
  griddep_wait();
  constexpr int K = MODE == 0 ? kF : 2 * kH;
  constexpr int SA = MODE == 0 ? kSX : kSA;
  constexpr int NR = MODE == 0 ? 1 : 8;          // 16-byte row pieces per thread
  constexpr int SO = kH + 8;                     // output tile row stride
  __shared__ __align__(16) __nv_bfloat16 sA[kTile * SA];
  __shared__ __align__(16) __nv_bfloat16 sB[kH * SA];
  __shared__ __align__(16) __nv_bfloat16 sO[MODE <= 1 ? kTile * SO : 8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // B^T[64 x K]
  if constexpr (MODE == 0) {
    for (int q = threadIdx.x; q < kH * kF / 8; q += blockDim.x)
      reinterpret_cast<uint4 *>(sB + (q / 2) * SA)[q & 1] = reinterpret_cast<const uint4 *>(a.wbf)[q];
  } else {
    const __nv_bfloat16 *w = a.wbf + kH * kF + (size_t)layer * kH * 2 * kH;   // [64][128] = [Ws | Wn]
    if constexpr (MODE == 1) {
      for (int q = threadIdx.x; q < kH * 2 * kH / 8; q += blockDim.x)
        reinterpret_cast<uint4 *>(sB + (q / 16) * SA)[q & 15] = reinterpret_cast<const uint4 *>(w)[q];
    } else {
      // dgrad: B[k][o] = Ws[k][o] (k < 64), Wn[k-64][o]; B^T[o][k]
      for (int q = threadIdx.x; q < kH * 2 * kH; q += blockDim.x) {
        const int o = q / (2 * kH), k = q % (2 * kH);
        sB[o * SA + k] = k < kH ? w[k * 2 * kH + o] : w[(k - kH) * 2 * kH + kH + o];
      }
    }
  }
  // Thread's pieces: mode 0, row tid/2, piece tid&1 of the 32-byte x row;
  // modes 1-2, rows tid/16 + 8k (k < 8), piece tid&15 of [self | message].
  const int piece = MODE == 0 ? (threadIdx.x & 1) : (threadIdx.x & 15);
  const int row0 = MODE == 0 ? (threadIdx.x >> 1) : (threadIdx.x >> 4);
  auto load = [&](int tile, uint4 (&r)[NR]) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const int i = tile * kTile + row0 + 8 * k;
      r[k] = make_uint4(0u, 0u, 0u, 0u);
      if (i >= a.n) continue;
      if constexpr (MODE == 0) {
        r[k] = reinterpret_cast<const uint4 *>(hin + (size_t)i * kF)[piece];
      } else if (piece >= 8) {
        r[k] = reinterpret_cast<const uint4 *>(msg + (size_t)i * kH)[piece - 8];
      } else if constexpr (MODE == 1) {
        r[k] = reinterpret_cast<const uint4 *>(hin + (size_t)i * kH)[piece];
      } else {
        const float4 *d = reinterpret_cast<const float4 *>(dzin + (size_t)i * kH) + 2 * piece;
        const float4 d0 = d[0], d1 = d[1];
        r[k] = make_uint4(pack_bf16(d0.x, d0.y), pack_bf16(d0.z, d0.w), pack_bf16(d1.x, d1.y),
                          pack_bf16(d1.z, d1.w));
      }
    }
  };
  uint4 r[NR];
  int tile = blockIdx.x;
  if (tile < ntiles) load(tile, r);
  const int g = lane >> 2, t = lane & 3;
  const float *bias = a.par + kOffLayer + layer * kLayerSz + 2 * kH * kH;
  for (; tile < ntiles; tile += gridDim.x) {
    const int node0 = tile * kTile;
    __syncthreads();                     // the previous tile is done with sA and sO
#pragma unroll
    for (int k = 0; k < NR; ++k) reinterpret_cast<uint4 *>(sA + (row0 + 8 * k) * SA)[piece] = r[k];
    __syncthreads();
    if (tile + (int)gridDim.x < ntiles) load(tile + gridDim.x, r);
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    warp_gemm_16x64<K>(sA + warp * 16 * SA, SA, sB, SA, acc);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int hlf = 0; hlf < 2; ++hlf) {
        const int row = warp * 16 + g + 8 * hlf, i = node0 + row;
        const int col = nt * 8 + 2 * t;
        float v0 = acc[nt][2 * hlf], v1 = acc[nt][2 * hlf + 1];
        if constexpr (MODE == 1) {
          v0 += bias[col];
          v1 += bias[col + 1];
        }
        if constexpr (MODE <= 1) {
          reinterpret_cast<unsigned *>(sO + row * SO + col)[0] = pack_bf16(fmaxf(v0, 0.f), fmaxf(v1, 0.f));
        } else {
          if (i >= a.n) continue;
          const float2 h = __bfloat1622float2(
              *reinterpret_cast<const __nv_bfloat162 *>(hin + (size_t)i * kH + col));
          reinterpret_cast<float2 *>(dzout + (size_t)i * kH + col)[0] =
              make_float2(h.x > 0.f ? v0 : 0.f, h.y > 0.f ? v1 : 0.f);
        }
      }
    if constexpr (MODE <= 1) {
      __syncthreads();
      for (int q = threadIdx.x; q < kTile * 8; q += blockDim.x) {
        const int row = q >> 3, i = node0 + row;
        if (i < a.n)
          reinterpret_cast<uint4 *>(hout + (size_t)i * kH)[q & 7] =
              reinterpret_cast<const uint4 *>(sO + row * SO)[q & 7];
      }
    }
  }
}

// Weight gradient partial of one CTA over its node chunks:
// P[o][k] = sum_i dz[i][o] A[i][k], A = [h | mean | 1] (K = 144) or [x]
// (K = 16, whose column 9 is the constant 1).  The mma's M is o (64), its
// N is k and its reduction runs over nodes.
template <int MODE>
__global__ void __launch_bounds__(kMpThreads) k_mp_wgrad(MpArgs a, const float *dz,
                                                          const __nv_bfloat16 *hin,
                                                          const __nv_bfloat16 *msg, float *part,
                                                          int chunks_per_cta) {
  griddep_wait();
  constexpr int K = MODE == 0 ? kF : 2 * kH + 16;
  constexpr int NT = K / 8;
  constexpr int SN = kTile + 8;   // node stride of the transposed tiles
  __shared__ __align__(16) __nv_bfloat16 sDt[kH * SN];    // dz^T [o][node]
  __shared__ __align__(16) __nv_bfloat16 sAt[K * SN];     // A^T [k][node]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
  for (int chunk = 0; chunk < chunks_per_cta; ++chunk) {
    const int node0 = (blockIdx.x * chunks_per_cta + chunk) * kTile;
    if (node0 >= a.n) break;
    __syncthreads();
    const int ch = threadIdx.x & 7;
    for (int r = threadIdx.x >> 3; r < kTile; r += kMpThreads / 8) {
      const int i = node0 + r;
      float d[8], self[8], agg[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) d[e] = self[e] = agg[e] = 0.f;
      if (i < a.n) {
        const float4 *dr = reinterpret_cast<const float4 *>(dz + (size_t)i * kH) + 2 * ch;
        const float4 d0 = dr[0], d1 = dr[1];
        d[0] = d0.x; d[1] = d0.y; d[2] = d0.z; d[3] = d0.w;
        d[4] = d1.x; d[5] = d1.y; d[6] = d1.z; d[7] = d1.w;
        if constexpr (MODE == 0) {
          if (ch < 2) unpack_bf16x8(self, reinterpret_cast<const uint4 *>(hin + (size_t)i * kF)[ch]);
        } else {
          unpack_bf16x8(self, reinterpret_cast<const uint4 *>(hin + (size_t)i * kH)[ch]);
          unpack_bf16x8(agg, reinterpret_cast<const uint4 *>(msg + (size_t)i * kH)[ch]);
        }
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) sDt[(8 * ch + e) * SN + r] = __float2bfloat16_rn(d[e]);
      if constexpr (MODE == 0) {
        if (ch < 2)
#pragma unroll
          for (int e = 0; e < 8; ++e) sAt[(8 * ch + e) * SN + r] = __float2bfloat16_rn(self[e]);
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          sAt[(8 * ch + e) * SN + r] = __float2bfloat16_rn(self[e]);
          sAt[(kH + 8 * ch + e) * SN + r] = __float2bfloat16_rn(agg[e]);
        }
        // the bias column (row 128 of A^T) and its zero padding
#pragma unroll
        for (int e = 0; e < 2; ++e)
          sAt[(2 * kH + 2 * ch + e) * SN + r] = __float2bfloat16_rn(ch == 0 && e == 0 && i < a.n ? 1.f : 0.f);
      }
    }
    __syncthreads();
    // warp w: rows o = 16 w .. 16 w + 15 of the partial, all K columns
    const __nv_bfloat16 *A = sDt + warp * 16 * SN;
#pragma unroll
    for (int k0 = 0; k0 < kTile; k0 += 16) {
      const unsigned a0 = *reinterpret_cast<const unsigned *>(A + g * SN + k0 + 2 * t);
      const unsigned a1 = *reinterpret_cast<const unsigned *>(A + (g + 8) * SN + k0 + 2 * t);
      const unsigned a2 = *reinterpret_cast<const unsigned *>(A + g * SN + k0 + 2 * t + 8);
      const unsigned a3 = *reinterpret_cast<const unsigned *>(A + (g + 8) * SN + k0 + 2 * t + 8);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const __nv_bfloat16 *b = sAt + (nt * 8 + g) * SN + k0 + 2 * t;
        mma_bf16(acc[nt], a0, a1, a2, a3, *reinterpret_cast<const unsigned *>(b),
                 *reinterpret_cast<const unsigned *>(b + 8));
      }
    }
  }
  float *pc = part + (size_t)blockIdx.x * kH * K;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int o = warp * 16 + g, k = nt * 8 + 2 * t;
    pc[o * K + k] = acc[nt][0];
    pc[o * K + k + 1] = acc[nt][1];
    pc[(o + 8) * K + k] = acc[nt][2];
    pc[(o + 8) * K + k + 1] = acc[nt][3];
  }
}

// Sums the CTA partials in CTA order into the gradient slots of one layer
// (mode 1: Ws, Wn, b) or of the input layer (mode 0: W_in).
__global__ void k_mp_wreduce(const float *part, int nctas, int mode, int layer, float *grad) {
  griddep_wait();
  const int K = mode == 0 ? kF : 2 * kH + 16;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kH * K) return;
  float s = 0.f;
  for (int b = 0; b < nctas; ++b) s += part[(size_t)b * kH * K + q];
  const int o = q / K, k = q % K;
  if (mode == 0) {
    grad[kOffWin + o * kF + k] = s;
    return;
  }
  float *gl = grad + kOffLayer + layer * kLayerSz;
  if (k < kH) gl[o * kH + k] = s;                       // Ws[o][k]
  else if (k < 2 * kH) gl[kH * kH + o * kH + (k - kH)] = s;   // Wn[o][k - 64]
  else if (k == 2 * kH) gl[2 * kH * kH + o] = s;        // b[o]
}

// ------------------------------------------------------------ the head
// out_i = w_out . h3_i + b_out; the guess at wet interior nodes, the
// reference elsewhere.  With `loss`, also dL/dout_i (Huber loss of the
// normalised correction over wet interior nodes, target from the solved
// ETAS) and the block partials of the loss.  8 lanes per node, 8 channels
// each.
constexpr int kHeadThreads = 256;

__host__ __device__ constexpr int head_blocks(int n) {
  return (int)(((long long)n * 8 + kHeadThreads - 1) / kHeadThreads);
}

__global__ void __launch_bounds__(kHeadThreads) k_mp_head(adc_ctx c, Mpnn m, int mode) {
  griddep_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x, i = q >> 3, ch = q & 7;
  float hv[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) hv[e] = 0.f;
  if (i < m.n) unpack_bf16x8(hv, reinterpret_cast<const uint4 *>(m.h[kL] + (size_t)i * kH)[ch]);
  const float *w = m.par + kOffWout + 8 * ch;
  float s = 0.f;
#pragma unroll
  for (int e = 0; e < 8; ++e) s += hv[e] * w[e];
  s += __shfl_xor_sync(0xffffffffu, s, 4);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  double l = 0.0;
  if (i < m.n && ch == 0) {
    const float out = s + m.par[kOffBout];
    const double s_out = (double)m.par[kOffNorm + 2 * kNF];
    const bool use = c.nodecode[i] == 1 && c.is_nbd[i] < 0;
    if (mode == 0) {
      m.pred[i] = use ? m.ref[i] + s_out * out : m.ref[i];
    } else {
      float d = 0.f;
      if (use) {
        const double sol = m.tgt ? m.tgt[i] : c.etas[i];
        const float tgt = (float)((sol - m.ref[i]) / s_out);
        const float e = out - tgt, ae = fabsf(e);
        d = fminf(fmaxf(e, -kHuber), kHuber);
        l = ae <= kHuber ? (double)e * e : (double)kHuber * (2.0 * ae - kHuber);
      }
      m.dout[i] = d;   // half the loss derivative; scaled by 2 / n in the backward pass
    }
  }
  if (mode == 1) {
    __shared__ double sh[kHeadThreads / 32];
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < kHeadThreads / 32; ++k) t += sh[k];
      m.loss_part[blockIdx.x] = t;
    }
  }
}

// dz3 = (dL/dout w_out) * (h3 > 0) with dL/dout = 2 clamp(e) / n (the loss
// is the mean over all nodes of the Huber loss of e, e = 0 where the guess
// is not used); 8 lanes per node.
__global__ void __launch_bounds__(kHeadThreads) k_mp_head_bwd(Mpnn m) {
  griddep_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x, i = q >> 3, ch = q & 7;
  if (i >= m.n) return;
  const float d = m.dout[i] * (2.f / (float)m.n);
  float hv[8];
  unpack_bf16x8(hv, reinterpret_cast<const uint4 *>(m.h[kL] + (size_t)i * kH)[ch]);
  const float *w = m.par + kOffWout + 8 * ch;
  float o[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) o[e] = hv[e] > 0.f ? d * w[e] : 0.f;
  float4 *dst = reinterpret_cast<float4 *>(m.dz[0] + (size_t)i * kH) + 2 * ch;
  dst[0] = make_float4(o[0], o[1], o[2], o[3]);
  dst[1] = make_float4(o[4], o[5], o[6], o[7]);
}

// Head gradient partials per CTA (its nodes, warp-strided, lanes over
// channel pairs): dw_out[k] = sum d_i h3_i[k], db_out = sum d_i, with
// d_i = 2 clamp(e_i) / n.  Row b of `part` holds CTA b's 65 sums.
__global__ void k_mp_head_grad(Mpnn m, int nodes_per_cta) {
  griddep_wait();
  __shared__ float sh[kMpThreads / 32][kH + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int i0 = blockIdx.x * nodes_per_cta, i1 = min(m.n, i0 + nodes_per_cta);
  float s0 = 0.f, s1 = 0.f, sb = 0.f;
  for (int i = i0 + warp; i < i1; i += nw) {
    const float d = m.dout[i] * (2.f / (float)m.n);
    const float2 h = __bfloat1622float2(reinterpret_cast<const __nv_bfloat162 *>(m.h[kL] + (size_t)i * kH)[lane]);
    s0 += d * h.x;
    s1 += d * h.y;
    sb += d;
  }
  sh[warp][2 * lane] = s0;
  sh[warp][2 * lane + 1] = s1;
  if (lane == 0) sh[warp][kH] = sb;
  __syncthreads();
  for (int k = threadIdx.x; k <= kH; k += blockDim.x) {
    float t = 0.f;
    for (int w = 0; w < nw; ++w) t += sh[w][k];
    m.part[(size_t)blockIdx.x * (kH + 1) + k] = t;
  }
}

// Sums the head partials in CTA order, and the loss partials of k_mp_head
// (fixed tree) into stats[0] (the mean Huber loss of the normalised error).
__global__ void k_mp_head_reduce(Mpnn m, int nctas, int nloss) {
  griddep_wait();
  __shared__ double sh[32];
  if (threadIdx.x <= kH) {
    float t = 0.f;
    for (int b = 0; b < nctas; ++b) t += m.part[(size_t)b * (kH + 1) + threadIdx.x];
    m.grad[threadIdx.x < kH ? kOffWout + threadIdx.x : kOffBout] = t;
  }
  double l = 0.0;
  for (int b = threadIdx.x; b < nloss; b += blockDim.x) l += m.loss_part[b];
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    m.stats[0] = t / (double)m.n;
  }
}

// Adam on the trained parameters; refreshes the BF16 weight copies.
__global__ void k_mp_adam(Mpnn m) {
  griddep_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const double step = m.stats[1] + 1.0;
  if (q < kNTrain) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gq = m.grad[q];
    const float m1 = b1 * m.m1[q] + (1.f - b1) * gq;
    const float m2 = b2 * m.m2[q] + (1.f - b2) * gq * gq;
    m.m1[q] = m1;
    m.m2[q] = m2;
    const float c1 = 1.f - (float)pow((double)b1, step), c2 = 1.f - (float)pow((double)b2, step);
    float p = m.par[q] - m.lr * (m1 / c1) / (sqrtf(m2 / c2) + eps);
    if (q >= kOffWin && q < kOffWin + kH * kF && (q % kF) > kNF) p = 0.f;   // padding stays 0
    m.par[q] = p;
  }
  if (q == 0) m.stats[1] = step;
}

// BF16 copies of the weight matrices: W_in [64][16], then per layer the
// rows [Ws[o][:] | Wn[o][:]] of 128.
__global__ void k_mp_tobf16(Mpnn m) {
  griddep_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < kH * kF) {
    m.wbf[q] = __float2bfloat16_rn(m.par[kOffWin + q]);
    return;
  }
  const int r = q - kH * kF;
  if (r >= kL * kH * 2 * kH) return;
  const int layer = r / (kH * 2 * kH), rem = r % (kH * 2 * kH), o = rem / (2 * kH), k = rem % (2 * kH);
  const float *pl = m.par + kOffLayer + layer * kLayerSz;
  const float v = k < kH ? pl[o * kH + k] : pl[kH * kH + o * kH + (k - kH)];
  m.wbf[q] = __float2bfloat16_rn(v);
}

static MpArgs mp_args(const Mpnn &m) {
  return MpArgs{m.n, m.wbf, m.par, m.nb_ptr, m.nb_idx, m.inv_deg};
}

// Forward pass: features, input layer, three message-passing layers (each
// a ring aggregation and a dense pass), head (the guess in m.pred).
int launch_predictor_forward(adc_ctx *c) {
  Mpnn *mp = c->mp;
  if (!mp || !(mp->learned || mp->train)) return ADC_OK;
  const Mpnn &m = *mp;
  const MpArgs a = mp_args(m);
  const int tiles = (m.n + kTile - 1) / kTile;
  const __nv_bfloat16 *none = nullptr;
  launch_k(k_mp_features, nblk(m.n), kThreads, c->stream, *c, m);
  launch_k(k_mp_dense<0>, std::min(tiles, m.dense_ctas[0]), kMpThreads, c->stream, a, 0,
           (const __nv_bfloat16 *)m.x, none, (const float *)nullptr, m.h[0], (float *)nullptr, tiles);
  for (int l = 0; l < kL; ++l) {
    launch_k(k_mp_aggr, tiles, kMpThreads, c->stream, a, (const __nv_bfloat16 *)m.h[l], m.mean[l]);
    launch_k(k_mp_dense<1>, std::min(tiles, m.dense_ctas[1]), kMpThreads, c->stream, a, l,
             (const __nv_bfloat16 *)m.h[l], (const __nv_bfloat16 *)m.mean[l], (const float *)nullptr,
             m.h[l + 1], (float *)nullptr, tiles);
  }
  launch_k(k_mp_head, head_blocks(m.n), kHeadThreads, c->stream, *c, m, 0);
  c->launches += 3 + 2 * kL;
  return ADC_OK;
}

// Loss and backpropagation for (the features of this step, the solved
// ETAS): the gradient of every trained parameter in m.grad.
static int launch_predictor_backward(adc_ctx *c) {
  const Mpnn &m = *c->mp;
  const MpArgs a = mp_args(m);
  const int tiles = (m.n + kTile - 1) / kTile;
  const int hb = head_blocks(m.n);
  launch_k(k_mp_head, hb, kHeadThreads, c->stream, *c, m, 1);
  launch_k(k_mp_head_bwd, hb, kHeadThreads, c->stream, m);
  const int npc = (m.n + m.part_ctas - 1) / m.part_ctas;
  launch_k(k_mp_head_grad, m.part_ctas, kMpThreads, c->stream, m, npc);
  launch_k(k_mp_head_reduce, 1, 1024, c->stream, m, m.part_ctas, hb);
  const int chunks = (tiles + m.part_ctas - 1) / m.part_ctas;
  int cur = 0;
  for (int l = kL - 1; l >= 0; --l) {
    // dz[cur] holds dz of layer l+1 (h_{l+1} = ReLU(z_{l+1}))
    launch_k(k_mp_wgrad<1>, m.part_ctas, kMpThreads, c->stream, a, (const float *)m.dz[cur],
             (const __nv_bfloat16 *)m.h[l], (const __nv_bfloat16 *)m.mean[l], m.part, chunks);
    launch_k(k_mp_wreduce, (kH * (2 * kH + 16) + 255) / 256, 256, c->stream,
             (const float *)m.part, m.part_ctas, 1, l, m.grad);
    launch_k(k_mp_aggr_dz, tiles, kMpThreads, c->stream, a, (const float *)m.dz[cur], m.adz);
    launch_k(k_mp_dense<2>, std::min(tiles, m.dense_ctas[2]), kMpThreads, c->stream, a, l,
             (const __nv_bfloat16 *)m.h[l], (const __nv_bfloat16 *)m.adz, (const float *)m.dz[cur],
             (__nv_bfloat16 *)nullptr, m.dz[cur ^ 1], tiles);
    cur ^= 1;
  }
  const __nv_bfloat16 *none = nullptr;
  launch_k(k_mp_wgrad<0>, m.part_ctas, kMpThreads, c->stream, a, (const float *)m.dz[cur],
           (const __nv_bfloat16 *)m.x, none, m.part, chunks);
  launch_k(k_mp_wreduce, (kH * kF + 255) / 256, 256, c->stream, (const float *)m.part,
           m.part_ctas, 0, 0, m.grad);
  c->launches += 4 + 4 * kL + 2;
  return ADC_OK;
}

// Training step: backpropagation, then Adam and the BF16 weight copies.
int launch_predictor_train(adc_ctx *c) {
  Mpnn *mp = c->mp;
  if (!mp || !mp->train) return ADC_OK;
  int rc = launch_predictor_backward(c);
  if (rc) return rc;
  launch_k(k_mp_adam, (kNTrain + 255) / 256, 256, c->stream, *mp);
  launch_k(k_mp_tobf16, (kH * kF + kL * kH * 2 * kH + 255) / 256, 256, c->stream, *mp);
  c->launches += 2;
  return ADC_OK;
}

// Builds the predictor state on first use: 1-ring CSR from the bound
// NeiTab, buffers, zeroed moments.
static int mp_alloc(adc_ctx *c) {
  if (c->mp) return ADC_OK;
  if (!c->h_neitab || !c->h_nneigh) {
    set_error("the predictor needs the bound NeiTab");
    return ADC_ERR_ARG;
  }
  const int n = c->np;
  std::vector<int> ptr(n + 1, 0), idx;
  std::vector<float> inv(n, 0.f);
  idx.reserve((size_t)n * 7);
  for (int i = 0; i < n; ++i) {
    const int nn = c->h_nneigh[i];
    for (int j = 2; j <= nn; ++j) {   // slot 1 is the node itself
      const int v = c->h_neitab[i + (size_t)n * (j - 1)];
      if (v >= 1 && v <= n && v - 1 != i) idx.push_back(v - 1);
    }
    ptr[i + 1] = (int)idx.size();
    const int deg = ptr[i + 1] - ptr[i];
    inv[i] = deg > 0 ? 1.f / (float)deg : 0.f;
  }
  Mpnn *m = new Mpnn();
  memset(m, 0, sizeof(*m));
  m->n = n;
  m->lr = 1e-3f;
  m->part_ctas = 4 * 148;
  {
    int dev = 0, sms = 148, per[3] = {1, 1, 1};
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0], k_mp_dense<0>, kMpThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1], k_mp_dense<1>, kMpThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[2], k_mp_dense<2>, kMpThreads, 0);
    for (int k = 0; k < 3; ++k) m->dense_ctas[k] = std::max(1, per[k]) * sms;
  }
  auto al = [&](auto **p, size_t cnt) -> int {
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(cnt, 1) * sizeof(**p));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (predictor)");
    return ADC_OK;
  };
  int rc = 0;
  rc |= al(&m->par, kNParams); rc |= al(&m->grad, kNParams);
  rc |= al(&m->m1, kNParams); rc |= al(&m->m2, kNParams);
  rc |= al(&m->wbf, (size_t)kH * kF + (size_t)kL * kH * 2 * kH);
  rc |= al(&m->x, (size_t)n * kF);
  for (int l = 0; l <= kL; ++l) rc |= al(&m->h[l], (size_t)n * kH);
  for (int l = 0; l < kL; ++l) rc |= al(&m->mean[l], (size_t)n * kH);
  rc |= al(&m->adz, (size_t)n * kH);
  rc |= al(&m->dz[0], (size_t)n * kH); rc |= al(&m->dz[1], (size_t)n * kH);
  rc |= al(&m->ref, n); rc |= al(&m->pred, n); rc |= al(&m->dout, n);
  rc |= al(&m->nb_ptr, n + 1); rc |= al(&m->nb_idx, idx.size()); rc |= al(&m->inv_deg, n);
  rc |= al(&m->part, (size_t)m->part_ctas * kH * (2 * kH + 16));
  rc |= al(&m->loss_part, (size_t)head_blocks(n) + 1);
  rc |= al(&m->stats, kNStats);
  if (rc) return ADC_ERR_NOMEM;
  ADC_CUDA(cudaMemcpy(m->nb_ptr, ptr.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (!idx.empty())
    ADC_CUDA(cudaMemcpy(m->nb_idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMemcpy(m->inv_deg, inv.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMemset(m->par, 0, kNParams * sizeof(float)));
  ADC_CUDA(cudaMemset(m->grad, 0, kNParams * sizeof(float)));
  ADC_CUDA(cudaMemset(m->m1, 0, kNParams * sizeof(float)));
  ADC_CUDA(cudaMemset(m->m2, 0, kNParams * sizeof(float)));
  ADC_CUDA(cudaMemset(m->stats, 0, kNStats * sizeof(double)));
  ADC_CUDA(cudaMemset(m->dz[0], 0, (size_t)n * kH * sizeof(float)));
  ADC_CUDA(cudaMemset(m->dz[1], 0, (size_t)n * kH * sizeof(float)));
  c->mp = m;
  return ADC_OK;
}

void mp_free(adc_ctx *c) {
  Mpnn *m = c->mp;
  if (!m) return;
  void *ptrs[] = {m->par, m->grad, m->m1, m->m2, m->wbf, m->x, m->h[0], m->h[1], m->h[2], m->h[3],
                  m->mean[0], m->mean[1], m->mean[2], m->adz, m->dz[0], m->dz[1], m->ref, m->pred, m->dout, m->nb_ptr, m->nb_idx, m->inv_deg,
                  m->part, m->loss_part, m->stats};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete m;
  c->mp = nullptr;
}

const double *mp_guess(const adc_ctx *c) {
  return (c->mp && c->mp->learned) ? c->mp->pred : nullptr;
}

}  // namespace adc

using namespace adc;

extern "C" {

int adc_predictor_nparams(void) { return kNParams; }

int adc_set_predictor(adc_ctx *c, const float *params, int nparams) {
  if (!c || !params || nparams != kNParams) {
    set_error("adc_set_predictor: expected %d parameters", kNParams);
    return ADC_ERR_ARG;
  }
  for (int k = 0; k < kNF; ++k)
    if (!(params[kOffNorm + kNF + k] > 0.f)) {
      set_error("adc_set_predictor: feature scale %d must be positive", k);
      return ADC_ERR_ARG;
    }
  if (!(params[kOffNorm + 2 * kNF] > 0.f)) {
    set_error("adc_set_predictor: output scale must be positive");
    return ADC_ERR_ARG;
  }
  int rc = mp_alloc(c);
  if (rc) return rc;
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  ADC_CUDA(cudaMemcpy(c->mp->par, params, kNParams * sizeof(float), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMemset(c->mp->m1, 0, kNParams * sizeof(float)));
  ADC_CUDA(cudaMemset(c->mp->m2, 0, kNParams * sizeof(float)));
  ADC_CUDA(cudaMemset(c->mp->stats, 0, kNStats * sizeof(double)));
  k_mp_tobf16<<<(kH * kF + kL * kH * 2 * kH + 255) / 256, 256, 0, c->stream>>>(*c->mp);
  ADC_CUDA(cudaGetLastError());
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  c->mp->learned = (c->prec & ADC_LEARNED_START) ? 1 : 0;
  drop_graphs(c);   // the step sequence changes
  return ADC_OK;
}

int adc_get_predictor(adc_ctx *c, float *params, int nparams) {
  if (!c || !params || nparams != kNParams || !c->mp) {
    set_error("adc_get_predictor: no predictor or wrong size (%d)", kNParams);
    return ADC_ERR_ARG;
  }
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  ADC_CUDA(cudaMemcpy(params, c->mp->par, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
  return ADC_OK;
}

int adc_predictor_train(adc_ctx *c, int on, float lr) {
  if (!c || !c->mp) {
    set_error("adc_predictor_train: set a predictor first");
    return ADC_ERR_ARG;
  }
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  c->mp->train = on ? 1 : 0;
  c->mp->lr = lr;
  drop_graphs(c);
  return ADC_OK;
}

int adc_predictor_stats(adc_ctx *c, double *loss, long long *adam_steps) {
  if (!c || !c->mp) return ADC_ERR_ARG;
  double s[kNStats];
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  ADC_CUDA(cudaMemcpy(s, c->mp->stats, sizeof(s), cudaMemcpyDeviceToHost));
  if (loss) *loss = s[0];
  if (adam_steps) *adam_steps = (long long)s[1];
  return ADC_OK;
}

int adc_predictor_forward(adc_ctx *c, double *guess, float *hidden3) {
  if (!c || !c->mp) return ADC_ERR_ARG;
  const int saved = c->mp->learned;
  c->mp->learned = 1;
  int rc = launch_predictor_forward(c);
  c->mp->learned = saved;
  if (rc) return rc;
  ADC_CUDA(cudaGetLastError());
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  if (guess) ADC_CUDA(cudaMemcpy(guess, c->mp->pred, c->np * sizeof(double), cudaMemcpyDeviceToHost));
  if (hidden3) {
    std::vector<__nv_bfloat16> h((size_t)c->np * kH);
    ADC_CUDA(cudaMemcpy(h.data(), c->mp->h[kL], h.size() * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < h.size(); ++q) hidden3[q] = __bfloat162float(h[q]);
  }
  return ADC_OK;
}

int adc_predictor_gradient_at(adc_ctx *c, const double *target, float *grad, int nparams) {
  if (!c || !c->mp || !target || !grad || nparams != kNParams) return ADC_ERR_ARG;
  double *d = nullptr;
  ADC_CUDA(cudaMalloc((void **)&d, c->np * sizeof(double)));
  cudaError_t e = cudaMemcpy(d, target, c->np * sizeof(double), cudaMemcpyHostToDevice);
  int rc = ADC_OK;
  if (e == cudaSuccess) {
    const int saved = c->mp->learned;
    c->mp->learned = 1;
    rc = launch_predictor_forward(c);
    c->mp->learned = saved;
    c->mp->tgt = d;
    if (!rc) rc = launch_predictor_backward(c);
    c->mp->tgt = nullptr;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(grad, c->mp->grad, kNParams * sizeof(float), cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "adc_predictor_gradient_at");
  return rc;
}

int adc_predictor_gradient(adc_ctx *c, float *grad, int nparams) {
  if (!c || !c->mp || !grad || nparams != kNParams) return ADC_ERR_ARG;
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  ADC_CUDA(cudaMemcpy(grad, c->mp->grad, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
  return ADC_OK;
}

}  // extern "C"
