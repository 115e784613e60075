// Register/shared-memory FFT building blocks for sm_100a.
//
// A length-L transform (L = E*T, E >= T, E % T == 0, both powers of two) is computed by T threads that each hold
// E complex values in registers:
//   stage 1  thread t holds x[t + T*e] (e < E), does an E-point DFT in registers and multiplies output k1 by
//            w_L^(t*k1) (table in shared memory, laid out [k1][t] so a warp reads it conflict-free);
//   exchange the E x T intermediate goes through a per-vector shared buffer with pitch T+1 (conflict-free for both
//            the column write and the row read);
//   stage 2  thread t takes k1 = t + T*m (m < E/T) and does T-point DFTs over the threads' values.
// On return thread t holds X[t + T*e] in register v[m*T + k2] with e = m + (E/T)*k2, i.e. the same index set
// it loaded, so transforms can be chained (forward -> pointwise -> inverse) with no data movement.
//
// The in-register DFTs are radix-2 decimation-in-frequency with compile-time twiddles (all indices resolve at
// compile time, so everything stays in registers); trivial twiddles (multiples of pi/4) skip the multiplies.
// Sign convention is cuFFT's: forward exp(-2*pi*i*k*n/L), inverse exp(+...), no scaling.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace pty {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
__device__ __forceinline__ float2 cconjmul(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// cos(2*pi*q/32) for q in [0, 8]: exact values of the first octant, rounded to float.
__host__ __device__ constexpr float cos32_octant(int q) {
  return q == 0 ? 1.0f
       : q == 1 ? 0.98078528040323044913f
       : q == 2 ? 0.92387953251128675613f
       : q == 3 ? 0.83146961230254523708f
       : q == 4 ? 0.70710678118654752440f
       : q == 5 ? 0.55557023301960222474f
       : q == 6 ? 0.38268343236508977173f
       : q == 7 ? 0.19509032201612826785f
                : 0.0f;
}
// cos and sin of 2*pi*q/32 for any q in [0, 32) by octant symmetry.
__host__ __device__ constexpr float cos32(int q) {
  return q <= 8 ? cos32_octant(q) : q <= 16 ? -cos32_octant(16 - q) : q <= 24 ? -cos32_octant(q - 16)
                                                                               : cos32_octant(32 - q);
}
__host__ __device__ constexpr float sin32(int q) { return cos32((q + 24) % 32); }

// v * exp(-2*pi*i*Q/32) (forward) or v * exp(+2*pi*i*Q/32) (inverse), Q a compile-time constant.
template <int Q, bool INV>
__device__ __forceinline__ float2 twiddle32(float2 v) {
  constexpr int q = Q % 32;
  if constexpr (q == 0) {
    return v;
  } else if constexpr (q == 16) {
    return make_float2(-v.x, -v.y);
  } else if constexpr (q == 8) {  // exp(-i*pi/2) = -i
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  } else if constexpr (q == 24) {  // exp(-i*3pi/2) = +i
    return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  } else {
    constexpr float c = cos32(q), s = sin32(q);
    // forward: (x + iy)(c - is) = (xc + ys) + i(yc - xs); inverse: (x + iy)(c + is)
    if constexpr (INV)
      return make_float2(v.x * c - v.y * s, v.y * c + v.x * s);
    else
      return make_float2(v.x * c + v.y * s, v.y * c - v.x * s);
  }
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).  Register-array indices computed from
// the loop constant are then constant expressions, so the arrays never fall back to local memory.
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }
__host__ __device__ constexpr int bitrev(int i, int n) {
  int r = 0;
  for (int b = 0; b < ilog2(n); ++b) r |= ((i >> b) & 1) << (ilog2(n) - 1 - b);
  return r;
}

// ---- compile-time radix-2 DIF DFT on a register array (output in bit-reversed order) -------------------
template <int LEN, int S, int J, bool INV, int E>
__device__ __forceinline__ void dif_butterflies(float2 (&a)[E]) {
  if constexpr (J < LEN / 2) {
    float2 u = a[S + J], w = a[S + J + LEN / 2];
    a[S + J] = cadd(u, w);
    a[S + J + LEN / 2] = twiddle32<J*(32 / LEN), INV>(csub(u, w));
    dif_butterflies<LEN, S, J + 1, INV>(a);
  }
}
template <int LEN, int S, bool INV, int E>
__device__ __forceinline__ void dif_blocks(float2 (&a)[E]) {
  if constexpr (S < E) {
    dif_butterflies<LEN, S, 0, INV>(a);
    dif_blocks<LEN, S + LEN, INV>(a);
  }
}
template <int LEN, bool INV, int E>
__device__ __forceinline__ void dif_stages(float2 (&a)[E]) {
  if constexpr (LEN >= 2) {
    dif_blocks<LEN, 0, INV>(a);
    dif_stages<LEN / 2, INV>(a);
  }
}
// In place: afterwards a[bitrev(k)] = sum_n a_in[n] w_E^(k*n).  E <= 32.
template <bool INV, int E>
__device__ __forceinline__ void dft_reg(float2 (&a)[E]) {
  static_assert(E >= 2 && E <= 32 && (E & (E - 1)) == 0, "register DFT size");
  dif_stages<E, INV>(a);
}

// Thread layout of a length-L transform: L = E*T with T lanes per vector and E values per lane.
// E >= T: stage 2 is M = E/T T-point DFTs per lane.  E < T (Q = T/E = 2): each T-point DFT of stage 2 is shared by
// a lane pair through one radix-2 DIF step (L = 512 uses a whole warp per row with 16 values per lane, which keeps
// registers low enough for several CTAs per SM).
__host__ __device__ constexpr int fft_lanes(int L) {
  return L == 1024 ? 32 : L == 512 ? 32 : L == 256 ? 16 : L == 128 ? 8 : L == 64 ? 8 : L == 32 ? 4 : 0;
}
template <int L>
struct FftShape {
  static constexpr int T = fft_lanes(L);
  static constexpr int E = L / T;                    // registers (complex) per lane
  static constexpr int M = E >= T ? E / T : 1;       // stage-2 DFTs per lane (E >= T)
  static constexpr int Q = E >= T ? 1 : T / E;       // lanes per stage-2 DFT (E < T)
  static constexpr int XCH = E * (T + 1);            // exchange buffer (float2) per vector
  static constexpr int RC = (256 / T < L) ? 256 / T : L;  // rows (vectors) of a row-transform CTA
  static constexpr int THREADS = RC * T;                   // its block size (<= 256)
  static_assert(T > 0, "unsupported FFT length");
  static_assert(Q == 1 || Q == 2, "stage-2 split supports lane pairs only");
};

// Twiddle table for stage 1: tw[k1*T + t] = exp(-2*pi*i*t*k1/L); filled by fill_twiddles (double precision).
template <int L>
__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* __restrict__ g_tw) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) s_tw[i] = g_tw[i];
}

// One length-L transform by T cooperating lanes of a warp (lane index `t` = 0..T-1).
// v: on entry v[e] = x[t + T*e]; on exit element t + T*e is in v[out_slot<L>(e)].
// xch: this vector's exchange buffer (XCH float2).  Ends with __syncwarp (xch reusable).
template <int L, bool INV>
__device__ __forceinline__ void fft_vec(float2 (&v)[FftShape<L>::E], int t, float2* xch, const float2* s_tw) {
  constexpr int T = FftShape<L>::T, E = FftShape<L>::E, M = FftShape<L>::M, Q = FftShape<L>::Q;
  dft_reg<INV>(v);
  static_for<0, E>([&](auto k1c) {
    constexpr int k1 = decltype(k1c)::value;
    constexpr int src = bitrev(k1, E);
    if constexpr (k1 == 0) {
      xch[t] = v[src];
    } else {
      float2 w = s_tw[k1 * T + t];
      if (INV) w.y = -w.y;
      xch[k1 * (T + 1) + t] = cmul(v[src], w);
    }
  });
  __syncwarp();
  if constexpr (Q == 1) {
    static_for<0, M>([&](auto mc) {
      constexpr int m = decltype(mc)::value;
      float2 c[T];
#pragma unroll
      for (int tt = 0; tt < T; ++tt) c[tt] = xch[(t + T * m) * (T + 1) + tt];
      dft_reg<INV>(c);
      static_for<0, T>([&](auto k2c) {
        constexpr int k2 = decltype(k2c)::value;
        v[m * T + k2] = c[bitrev(k2, T)];
      });
    });
  } else {
    // lane t = k1 + E*q: radix-2 DIF over the two halves of the T-point DFT for its k1, keeping half q:
    // c[t'] = (b[t'] + (-1)^q b[t'+E]) * w_T^(q t'), then an E-point DFT gives outputs k2 = q + 2j.
    const int k1 = t % E;
    const bool odd = t >= E;
    const float sgn = odd ? -1.f : 1.f;
    const float2* row = xch + k1 * (T + 1);
    float2 c[E];
    static_for<0, E>([&](auto tc) {
      constexpr int tp = decltype(tc)::value;
      const float2 b0 = row[tp], b1 = row[tp + E];
      const float2 d = make_float2(b0.x + sgn * b1.x, b0.y + sgn * b1.y);
      const float2 dw = twiddle32<tp*(32 / T), INV>(d);
      c[tp] = odd ? dw : d;
    });
    dft_reg<INV>(c);
    static_for<0, E>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      v[j] = c[bitrev(j, E)];
    });
  }
  __syncwarp();
}

// ---- column transforms across a CTA ----------------------------------------------------------------------
// A CTA of T*CB threads transforms CB adjacent columns of a row-major L x L plane along the first index.
// Thread (s, c) holds column c at rows s + T*e (e < E), so every register load or store of the CTA touches CB
// consecutive elements of 32/CB rows (coalesced) and stage 1 (E-point DFT over e) needs no data movement; the
// exchange between the stages goes through `xch` (E x PK float2, PK = T*CB + 8: conflict-free for the stage-1
// writes and the stage-2 reads).  The stage-1 twiddle depends on s only.  On return the thread holds the transform
// at rows s + T*e in v[out_slot<L>(e)], the same index set it loaded, so forward -> pointwise -> inverse chains
// with no extra data movement.  Starts with __syncthreads (so xch may be reused back to back); a caller that
// reuses xch for anything else syncs first.
template <int L>
__host__ __device__ constexpr int cols_per_block() {
  return FftShape<L>::T == 32 ? 8 : FftShape<L>::T == 16 ? 16 : (L < 32 ? L : 32);
}
template <int L>
__host__ __device__ constexpr int cols_pitch() {
  return FftShape<L>::T * cols_per_block<L>() + 8;
}
template <int L>
__host__ __device__ constexpr int cols_threads() {
  return FftShape<L>::T * cols_per_block<L>();
}
template <int L>
__host__ __device__ constexpr int cols_xch_elems() {
  return FftShape<L>::E * cols_pitch<L>();
}

// Thread -> (s, c) of a column CTA: c fastest, so a warp covers 32/CB values of s (for T = 32 all on the same side
// of the stage-2 lane pairs, which keeps the pair branch warp-uniform and the twiddle reads contiguous).
template <int L>
__device__ __forceinline__ void cols_thread(int tid, int& s, int& c) {
  constexpr int CB = cols_per_block<L>();
  c = tid % CB;
  s = tid / CB;
}

template <int L, bool INV>
__device__ __forceinline__ void fft_cols(float2 (&v)[FftShape<L>::E], int s, int c, float2* xch,
                                         const float2* s_tw) {
  constexpr int T = FftShape<L>::T, E = FftShape<L>::E, M = FftShape<L>::M, Q = FftShape<L>::Q;
  constexpr int CB = cols_per_block<L>(), PK = cols_pitch<L>();
  dft_reg<INV>(v);
  __syncthreads();  // previous readers of xch are done
  static_for<0, E>([&](auto k1c) {
    constexpr int k1 = decltype(k1c)::value;
    constexpr int src = bitrev(k1, E);
    if constexpr (k1 == 0) {
      xch[s * CB + c] = v[src];
    } else {
      float2 w = s_tw[k1 * T + s];
      if (INV) w.y = -w.y;
      xch[k1 * PK + s * CB + c] = cmul(v[src], w);
    }
  });
  __syncthreads();
  if constexpr (Q == 1) {
    static_for<0, M>([&](auto mc) {
      constexpr int m = decltype(mc)::value;
      const float2* col = xch + (s + T * m) * PK + c;
      float2 a[T];
#pragma unroll
      for (int tt = 0; tt < T; ++tt) a[tt] = col[tt * CB];
      dft_reg<INV>(a);
      static_for<0, T>([&](auto k2c) {
        constexpr int k2 = decltype(k2c)::value;
        v[m * T + k2] = a[bitrev(k2, T)];
      });
    });
  } else {
    // s = k1 + E*q: radix-2 DIF over the two halves of the T-point DFT of k1, keeping half q (as in fft_vec)
    const int k1 = s % E;
    const bool odd = s >= E;
    const float sgn = odd ? -1.f : 1.f;
    const float2* col = xch + k1 * PK + c;
    float2 a[E];
    static_for<0, E>([&](auto tc) {
      constexpr int tp = decltype(tc)::value;
      const float2 b0 = col[tp * CB], b1 = col[(tp + E) * CB];
      const float2 d = make_float2(b0.x + sgn * b1.x, b0.y + sgn * b1.y);
      const float2 dw = twiddle32<tp*(32 / T), INV>(d);
      a[tp] = odd ? dw : d;
    });
    dft_reg<INV>(a);
    static_for<0, E>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      v[j] = a[bitrev(j, E)];
    });
  }
}

// Register slot of element index n = t + T*e for this lane after fft_vec.
template <int L>
__host__ __device__ constexpr int out_slot(int e) {
  return FftShape<L>::Q > 1 ? e : (e % FftShape<L>::M) * FftShape<L>::T + (e / FftShape<L>::M);
}

// After fft_vec the lane holds element t + T*e in v[out_slot(e)].  To feed a second transform (which wants
// v[e] = element t + T*e) reorder the registers (free at compile time).
template <int L>
__device__ __forceinline__ void to_input_order(float2 (&v)[FftShape<L>::E]) {
  constexpr int E = FftShape<L>::E;
  float2 tmp[E];
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    tmp[e] = v[out_slot<L>(e)];
  });
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = tmp[e];
}

}  // namespace pty
