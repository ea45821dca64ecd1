// Device-side bit_pack codec for sm_100a.
//
// A particle record is a little-endian bit stream over 64-bit words; slot s
// occupies bits [bit_offset, bit_offset + bits) and may straddle two words
// (reference: struct_llvm.cpp:77-116, codegen_llvm_quant.cpp:834-952).
// Quantized types follow the reference's arithmetic exactly:
//   fixed  encode  q = FPToSI(round((v - offset) * fl(1/scale) [+ u - 0.5]))
//                  (codegen_llvm_quant.cpp:44-80, runtime.cpp:1732-1762),
//                  code = q & mask(bits) (:166-184)
//          decode  v = float(sext(code)) * scale + offset (:624-641)
//   float with own exponent (:229-305, :660-757)
//   float with shared exponent (:347-499, :660-757)
// Every float operation is written with an explicit rounding intrinsic so
// that nvcc cannot contract it into an FMA, which would change the codes.
#pragma once

#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>
#endif

#include "../../include/aq.h"

namespace aq {

// ------------------------------------------------------------------ RNG
// Counter-based uniform per (seed, step, particle id, slot): SplitMix64
// finalizer (Steele, Lea & Flood 2014) for the per-step and per-particle
// keys; draw j of a particle is element j + 1 of the 32-bit LCG
// x' = 747796405 x + 2891336453 (the PCG multiplier; full period) started at
// the key's low half, reached in one multiply-add with jump constants known
// at compile time, then x ^ (x >> 16) ^ (high half of the key).  The
// reference's generator is a per-thread xorshift128 (runtime.cpp:522-536,
// 1560-1589) whose stream depends on the thread schedule; this one is
// reproducible.

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// LCG jump constants: element n of the sequence from x0 is A[n] x0 + C[n]
constexpr int AQ_LCG_JUMPS = 2 * AQ_MAX_SLOTS + 1;
struct LcgJumps {
  uint32_t a[AQ_LCG_JUMPS], c[AQ_LCG_JUMPS];
};
__host__ __device__ constexpr LcgJumps make_lcg_jumps() {
  LcgJumps t{};
  uint32_t a = 1u, c = 0u;
  for (int n = 0; n < AQ_LCG_JUMPS; ++n) {
    t.a[n] = a;
    t.c[n] = c;
    a *= 747796405u;
    c = c * 747796405u + 2891336453u;
  }
  return t;
}
__device__ constexpr LcgJumps kLcgJumps = make_lcg_jumps();

__host__ __device__ __forceinline__ uint64_t step_key(uint64_t seed, int64_t step) {
  return mix64(seed + (uint64_t)(step + 1) * 0xD1B54A32D192ED03ull);
}

__device__ __forceinline__ uint64_t particle_key(uint64_t sk, int32_t pid) {
  return mix64(sk ^ ((uint64_t)(uint32_t)pid * 0x9E3779B97F4A7C15ull));
}

__device__ __forceinline__ uint32_t draw32(uint64_t pk, uint32_t j) {
  const uint32_t x = kLcgJumps.a[j + 1u] * (uint32_t)pk + kLcgJumps.c[j + 1u];
  return x ^ (x >> 16) ^ (uint32_t)(pk >> 32);
}

// rand_f32 / rand_f64 of runtime.cpp:1579-1585: u32 * 2^-32, u64 * 2^-64
__device__ __forceinline__ float uniform_f32(uint64_t pk, int s) {
  return __fmul_rn(__uint2float_rn(draw32(pk, 2u * (uint32_t)s)), 2.3283064365386963e-10f);
}

__device__ __forceinline__ double uniform_f64(uint64_t pk, int s) {
  uint64_t u = ((uint64_t)draw32(pk, 2u * (uint32_t)s) << 32) | draw32(pk, 2u * (uint32_t)s + 1u);
  return __dmul_rn(__ull2double_rn(u), 5.421010862427522e-20);
}

// ------------------------------------------------------------ bit access

// w: the record's words, a pointer or a view with operator[] (GRec)
template <class WP>
__device__ __forceinline__ uint64_t get_bits(const WP& w, int off, int nb) {
  const int wi = off >> 6, sh = off & 63;
  uint64_t v = w[wi] >> sh;
  if (sh + nb > 64) v |= w[wi + 1] << (64 - sh);
  return nb < 64 ? (v & ((1ull << nb) - 1ull)) : v;
}

__device__ __forceinline__ int32_t sext32(uint32_t code, int nb) {
  const int sh = 32 - nb;
  return sh ? ((int32_t)(code << sh)) >> sh : (int32_t)code;
}

// Sequential writer of a record: fields arrive in bit order, whole words
// are emitted as they fill (the carry logic of BitPackAssignStmt,
// codegen_llvm_quant.cpp:919-947).  Unlike the reference it writes no word
// past the record when the last field ends exactly on a word boundary.
struct BitWriter {
  uint64_t acc;
  int fill;
  int wi;
  uint64_t* out;
  __device__ __forceinline__ explicit BitWriter(uint64_t* o) : acc(0), fill(0), wi(0), out(o) {}
  __device__ __forceinline__ void put(uint64_t code, int nb) {
    acc |= code << fill;
    const int nf = fill + nb;
    if (nf >= 64) {
      out[wi++] = acc;
      acc = nf > 64 ? (code >> (64 - fill)) : 0ull;
      fill = nf - 64;
    } else {
      fill = nf;
    }
  }
  __device__ __forceinline__ void flush() {
    if (fill > 0) out[wi++] = acc;
  }
};

// ----------------------------------------------------------- fixed point

template <class R>
__device__ __forceinline__ R dequant_fixed(const aq_slot& S, bool f64, uint32_t code) {
  // adding a zero offset is skipped: q * scale is never -0, so it is exact
  if (f64) {
    double q = S.is_signed ? (double)sext32(code, S.bits) : (double)code;
    const double y = __dmul_rn(q, S.scale_f64);
    return (R)(S.offset_f64 != 0.0 ? __dadd_rn(y, S.offset_f64) : y);
  }
  float q = S.is_signed ? __int2float_rn(sext32(code, S.bits)) : __uint2float_rn(code);
  const float y = __fmul_rn(q, S.scale_f32);
  return (R)(S.offset_f32 != 0.0f ? __fadd_rn(y, S.offset_f32) : y);
}

// u is the dithering uniform in the compute type (ignored unless dith).
__device__ __forceinline__ uint32_t quant_fixed_f32(const aq_slot& S, bool dith, float v, float u) {
  // v - 0 == v exactly (also for -0 and NaN): a zero offset is skipped
  float c = __fmul_rn(S.offset_f32 != 0.0f ? __fsub_rn(v, S.offset_f32) : v, S.inv_scale_f32);
  if (dith) c = __fsub_rn(__fadd_rn(c, u), 0.5f);
  c = __fadd_rn(c, copysignf(0.5f, c));
  uint32_t q = S.is_signed ? (uint32_t)__float2int_rz(c) : __float2uint_rz(c);
  return S.bits < 32 ? (q & ((1u << S.bits) - 1u)) : q;
}

__device__ __forceinline__ uint32_t quant_fixed_f64(const aq_slot& S, bool dith, double v, double u) {
  double c = __dmul_rn(S.offset_f64 != 0.0 ? __dsub_rn(v, S.offset_f64) : v, S.inv_scale_f64);
  if (dith) c = __dsub_rn(__dadd_rn(c, u), 0.5);
  c = __dadd_rn(c, copysign(0.5, c));
  uint32_t q = S.is_signed ? (uint32_t)__double2int_rz(c) : __double2uint_rz(c);
  return S.bits < 32 ? (q & ((1u << S.bits) - 1u)) : q;
}

// ------------------------------------------------- floats with exponents

__device__ __forceinline__ int conv_offset(int ebits) { return 127 - (1 << (ebits - 1)) + 1; }

__device__ __forceinline__ void quant_float_exp(const aq_slot& S, float v, uint32_t& dcode, uint32_t& ecode) {
  const int db = S.bits - S.is_signed;
  uint32_t fb = __float_as_uint(v);
  if (db < 23) fb += 1u << (22 - db);
  const uint32_t ex = (fb >> 23) & 0xffu;
  const uint32_t vb = (uint32_t)(((int32_t)fb) >> (23 - db));
  uint32_t digits = vb & ((1u << db) - 1u);
  if (S.is_signed) digits |= (fb & 0x80000000u) >> (31 - db);
  int e = (int)ex - (ex != 0 ? conv_offset(S.exp_bits) : 0);
  e = e < 0 ? 0 : e;
  ecode = (uint32_t)e & ((1u << S.exp_bits) - 1u);
  dcode = e != 0 ? digits : 0u;
}

__device__ __forceinline__ float dequant_float_exp(const aq_slot& S, uint32_t d, uint32_t E) {
  const int db = S.bits - S.is_signed;
  int eo = conv_offset(S.exp_bits);
  if (S.exp_bits < 8) eo = E != 0 ? eo : 0;
  uint32_t digits = (d & ((1u << S.bits) - 1u)) << (23 - db);
  uint32_t fb = ((E + (uint32_t)eo) << 23) | (digits & 0x7fffffu);
  if (S.is_signed) fb |= (digits & (1u << 23)) << 8;
  return __uint_as_float(fb);
}

__device__ __forceinline__ uint32_t shared_exp_code(int ebits, uint32_t max_exp) {
  int e = (int)max_exp - (max_exp != 0 ? conv_offset(ebits) : 0);
  e = e < 0 ? 0 : e;
  return (uint32_t)e & ((1u << ebits) - 1u);
}

__device__ __forceinline__ uint32_t quant_shared(const aq_slot& S, float v, uint32_t max_exp) {
  const int db = S.bits - S.is_signed;
  const uint32_t fb = __float_as_uint(v);
  const uint32_t ex = (fb >> 23) & 0xffu;
  const uint32_t sh = min(max_exp - ex, 31u);
  uint32_t digits = ((fb & 0x7fffffu) | (1u << 23)) >> sh;
  const int rs = 23 + S.is_signed - db + (S.is_signed ? 0 : 1);
  digits = min(digits + (1u << (rs - 1)), (1u << 24) - 1u) >> rs;
  if (S.is_signed) digits |= (fb & 0x80000000u) >> (31 - db);
  return digits;
}

__device__ __forceinline__ float dequant_shared(const aq_slot& S, uint32_t d_in, uint32_t E) {
  const int db = S.bits - S.is_signed;
  int eo = conv_offset(S.exp_bits);
  if (S.exp_bits < 8) eo = E != 0 ? eo : 0;
  uint32_t digits = d_in & ((1u << S.bits) - 1u);
  uint32_t sign = 0;
  if (S.is_signed) {
    sign = digits & (1u << db);
    digits ^= sign;
    sign <<= (31 - db);
    digits <<= 1;
  }
  const int extra = (31 - db) - __clz(digits);
  eo += extra + (S.is_signed ? 0 : 1);
  const int dshift = (23 - db) - extra;
  digits = dshift >= 32 ? 0u : (digits << dshift);
  uint32_t fb = ((E + (uint32_t)eo) << 23) | (digits & 0x7fffffu);
  if (E == 0 || d_in == 0) fb = 0;
  return __uint_as_float(fb | sign);
}

// ------------------------------------------------ record storage in HBM
// The simulator keeps its records in groups of 32 (records 32 g .. 32 g + 31,
// in the simulator's order): a group stores its words as pairs, pair j
// (words 2j and 2j+1) of all 32 records side by side, 16 bytes per record,
// then, for an odd word count, the last word of all 32 records, 8 bytes
// each.  Group g starts at word 32 g W, so every pair is 16-byte aligned,
// and a warp that reads 32 consecutive records loads each pair with one
// coalesced access of 16-byte vectors (512 contiguous bytes, or two runs
// when the records straddle a group boundary).  Buffers hold whole groups.
// aq_encode, aq_decode and the words exchanged through the C ABI keep each
// record's words contiguous, as the reference's bit_pack does.
__host__ __device__ __forceinline__ int64_t grec_word(int64_t r, int k, int W) {
  const int64_t base = (r >> 5) * 32 * (int64_t)W;
  const int l = (int)(r & 31), W2 = W & ~1;
  return k < W2 ? base + (int64_t)(k >> 1) * 64 + 2 * l + (k & 1) : base + (int64_t)W2 * 32 + l;
}

// words a grouped buffer of n records occupies
__host__ __device__ __forceinline__ int64_t grouped_words(int64_t n, int W) { return ((n + 31) >> 5) * 32 * (int64_t)W; }

// read view of record r of a grouped buffer (word index -> word)
struct GRec {
  const uint64_t* w;
  int64_t r;
  int W;
  __device__ __forceinline__ uint64_t operator[](int k) const { return w[grec_word(r, k, W)]; }
};

// Record r's W words into rec[0, W) / from rec: the pairs as 16-byte
// vectors.  WC: the word count when it is a compile-time constant, else 0.
template <int WC>
__device__ __forceinline__ void load_grec(const uint64_t* __restrict__ words, int64_t r, int W, uint64_t* rec) {
  const int Wn = WC ? WC : W, W2 = Wn & ~1;
  const uint64_t* g = words + (r >> 5) * 32 * (int64_t)Wn;
  const int l = (int)(r & 31);
#pragma unroll
  for (int k = 0; k < W2; k += 2) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(g + (k >> 1) * 64 + 2 * l));
    rec[k] = v.x;
    rec[k + 1] = v.y;
  }
  if (Wn & 1) rec[W2] = __ldg(g + W2 * 32 + l);
}

template <int WC>
__device__ __forceinline__ void store_grec(uint64_t* __restrict__ words, int64_t r, int W, const uint64_t* rec) {
  const int Wn = WC ? WC : W, W2 = Wn & ~1;
  uint64_t* g = words + (r >> 5) * 32 * (int64_t)Wn;
  const int l = (int)(r & 31);
#pragma unroll
  for (int k = 0; k < W2; k += 2) *reinterpret_cast<ulonglong2*>(g + (k >> 1) * 64 + 2 * l) = make_ulonglong2(rec[k], rec[k + 1]);
  if (Wn & 1) g[W2 * 32 + l] = rec[W2];
}

// --------------------------------------------------------------- records

// Decode slots [0, NS) (predicated on n_slots) from record w; slots whose
// bit is clear in MASK are left untouched.
template <int NS, class R, unsigned MASK = 0xffffffffu, class WP>
__device__ __forceinline__ void decode_record(const aq_layout& L, const WP& w, R (&vals)[NS]) {
  const bool f64 = L.compute_f64 != 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s >= L.n_slots) break;
    if (!((MASK >> s) & 1u)) continue;
    const aq_slot& S = L.slot[s];
    const uint64_t code = get_bits(w, S.bit_offset, S.bits);
    R v;
    switch (S.kind) {
      case AQ_FIXED:
        v = dequant_fixed<R>(S, f64, (uint32_t)code);
        break;
      case AQ_INT:
        v = S.is_signed ? (R)sext32((uint32_t)code, S.bits) : (R)(uint32_t)code;
        break;
      case AQ_FLOAT_EXP:
        v = (R)dequant_float_exp(S, (uint32_t)code, (uint32_t)get_bits(w, S.exp_offset, S.exp_bits));
        break;
      case AQ_SHARED_EXP:
        v = (R)dequant_shared(S, (uint32_t)code, (uint32_t)get_bits(w, S.exp_offset, S.exp_bits));
        break;
      case AQ_RAW_F32:
        v = (R)__uint_as_float((uint32_t)code);
        break;
      default:
        v = (R)__longlong_as_double((long long)code);
        break;
    }
    vals[s] = v;
  }
}

// Decode one slot (runtime index).
template <class R, class WP>
__device__ __forceinline__ R decode_slot(const aq_layout& L, int s, const WP& w) {
  const aq_slot& S = L.slot[s];
  const uint64_t code = get_bits(w, S.bit_offset, S.bits);
  switch (S.kind) {
    case AQ_FIXED:
      return dequant_fixed<R>(S, L.compute_f64 != 0, (uint32_t)code);
    case AQ_INT:
      return S.is_signed ? (R)sext32((uint32_t)code, S.bits) : (R)(uint32_t)code;
    case AQ_FLOAT_EXP:
      return (R)dequant_float_exp(S, (uint32_t)code, (uint32_t)get_bits(w, S.exp_offset, S.exp_bits));
    case AQ_SHARED_EXP:
      return (R)dequant_shared(S, (uint32_t)code, (uint32_t)get_bits(w, S.exp_offset, S.exp_bits));
    case AQ_RAW_F32:
      return (R)__uint_as_float((uint32_t)code);
    default:
      return (R)__longlong_as_double((long long)code);
  }
}

// Encode vals into record `out` (sequential word writes) and replace each
// value by its dequantized form, which is what a later read of the record
// returns.  pk: particle key for dithering; uf/ud: explicit uniforms (slot
// indexed, compute type) or null.
template <int NS, class R>
__device__ __forceinline__ void encode_record(const aq_layout& L, R (&vals)[NS], uint64_t* out, uint64_t pk,
                                              const float* uf, const double* ud) {
  const bool f64 = L.compute_f64 != 0;
  const bool dith = L.use_dithering != 0;
  uint32_t gmax[AQ_MAX_GROUPS];
#pragma unroll
  for (int g = 0; g < AQ_MAX_GROUPS; ++g) gmax[g] = 0;
  if (L.n_groups > 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (s >= L.n_slots) break;
      if (L.slot[s].kind == AQ_SHARED_EXP) {
        const uint32_t ex = (__float_as_uint((float)vals[s]) >> 23) & 0xffu;
        const int g = L.slot[s].group;
#pragma unroll
        for (int k = 0; k < AQ_MAX_GROUPS; ++k)
          if (g == k) gmax[k] = max(gmax[k], ex);
      }
    }
  }
  BitWriter bw(out);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s >= L.n_slots) break;
    const aq_slot& S = L.slot[s];
    const R v = vals[s];
    switch (S.kind) {
      case AQ_FIXED: {
        uint32_t q;
        if (f64) {
          double u = 0.0;
          if (dith) u = ud ? ud[s] : uniform_f64(pk, s);
          q = quant_fixed_f64(S, dith, (double)v, u);
        } else {
          float u = 0.0f;
          if (dith) u = uf ? uf[s] : uniform_f32(pk, s);
          q = quant_fixed_f32(S, dith, (float)v, u);
        }
        bw.put(q, S.bits);
        vals[s] = dequant_fixed<R>(S, f64, q);
        break;
      }
      case AQ_INT: {
        uint32_t q = S.is_signed ? (uint32_t)__double2int_rz((double)v) : __double2uint_rz((double)v);
        if (S.bits < 32) q &= (1u << S.bits) - 1u;
        bw.put(q, S.bits);
        vals[s] = S.is_signed ? (R)sext32(q, S.bits) : (R)q;
        break;
      }
      case AQ_FLOAT_EXP: {
        uint32_t d, e;
        quant_float_exp(S, (float)v, d, e);
        bw.put(e, S.exp_bits);
        bw.put(d, S.bits);
        vals[s] = (R)dequant_float_exp(S, d, e);
        break;
      }
      case AQ_SHARED_EXP: {
        uint32_t mx = 0;
#pragma unroll
        for (int k = 0; k < AQ_MAX_GROUPS; ++k)
          if (S.group == k) mx = gmax[k];
        const uint32_t e = shared_exp_code(S.exp_bits, mx);
        if (S.exp_first) bw.put(e, S.exp_bits);
        const uint32_t d = quant_shared(S, (float)v, mx);
        bw.put(d, S.bits);
        vals[s] = (R)dequant_shared(S, d, e);
        break;
      }
      case AQ_RAW_F32: {
        const float f = (float)v;
        bw.put(__float_as_uint(f), 32);
        vals[s] = (R)f;
        break;
      }
      default: {
        const double f = (double)v;
        bw.put((uint64_t)__double_as_longlong(f), 64);
        vals[s] = (R)f;
        break;
      }
    }
  }
  bw.flush();
}

}  // namespace aq
