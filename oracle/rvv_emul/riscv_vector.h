// riscv_vector.h — test infrastructure only (oracle side).
//
// A scalar stand-in for the RISC-V Vector C intrinsics (RVV 1.0 intrinsic
// API, the non-overloaded `__riscv_*` names) restricted to the operations
// that the reference's RVV kernels use: src/rvv/*.cpp of RVVLASparse (the
// CSR5, VNEC and VHCC kernels, which exist only in that form, and the RVV
// versions of the CRS, HCSR, SELL-C-sigma, LAV and CVR products).  With it
// those files compile unmodified for x86-64 (oracle/Makefile target
// `ref-rvv`), so the oracle's restatements can be checked against the
// reference's own code.  Nothing in the product path
// includes this header.
//
// Model: VLEN = RVV_EMUL_VLEN bits (default 256, the machine the reference's
// kernels are written for: VHCC keeps an 8-bit scan mask per fp64 vector of
// e64m2, VNEC uses 8 fp64 / 16 fp32 lanes).  A vector of SEW-bit elements at
// LMUL holds VLEN * LMUL / SEW elements; a mask vboolN_t holds VLEN / N
// elements, stored one byte per element here and as bit i of the register
// (LSB first) where a mask is reinterpreted from an integer vector.
// Semantics follow the intrinsic specification: `vl` elements are active;
// `_mu` keeps the maskedoff operand where the mask is 0; `_tu` keeps the
// destination's tail; `_m` (mask agnostic) leaves inactive elements 0;
// unordered reductions (vfredusum) add in element order; vfmacc/vfmadd are
// fused (one rounding, std::fma); indexed loads and stores take byte
// offsets.  Elements past `vl` of a result with no destination operand keep
// the first vector operand's values (tail agnostic).  A `vl` above VLMAX
// acts as an AVL and is clamped to VLMAX (see rve::avl).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

#ifndef RVV_EMUL_VLEN
#define RVV_EMUL_VLEN 256
#endif

template <class T, size_t N>
struct rve_v {
  T e[N];
};
template <size_t N>
struct rve_b {
  uint8_t e[N];
};

namespace rve {
// An intrinsic's vl is the AVL of the vsetvli the compiler emits for it: the
// operation runs on min(AVL, VLMAX) elements (the rule of common
// implementations; the specification allows any vl in [ceil(AVL/2), VLMAX]
// when AVL < 2 VLMAX), so a vl above VLMAX is clamped, never used as is.
inline size_t avl(size_t vl, size_t vlmax) { return vl < vlmax ? vl : vlmax; }
template <class V>
constexpr size_t lanes() { return sizeof(V{}.e) / sizeof(V{}.e[0]); }
template <class T>
inline T ld(const void* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}
template <class T>
inline void st(void* p, T v) { std::memcpy(p, &v, sizeof(T)); }
}  // namespace rve

#define RVE_N(SEW, NUM, DEN) ((size_t)(RVV_EMUL_VLEN) * (NUM) / (DEN) / (SEW))

typedef rve_v<double, RVE_N(64, 1, 1)> vfloat64m1_t;
typedef rve_v<double, RVE_N(64, 2, 1)> vfloat64m2_t;
typedef rve_v<double, RVE_N(64, 4, 1)> vfloat64m4_t;
typedef rve_v<double, RVE_N(64, 8, 1)> vfloat64m8_t;
typedef rve_v<float, RVE_N(32, 1, 1)> vfloat32m1_t;
typedef rve_v<float, RVE_N(32, 2, 1)> vfloat32m2_t;
typedef rve_v<float, RVE_N(32, 4, 1)> vfloat32m4_t;
typedef rve_v<float, RVE_N(32, 8, 1)> vfloat32m8_t;
typedef rve_v<uint32_t, RVE_N(32, 1, 2)> vuint32mf2_t;
typedef rve_v<uint32_t, RVE_N(32, 1, 1)> vuint32m1_t;
typedef rve_v<uint32_t, RVE_N(32, 2, 1)> vuint32m2_t;
typedef rve_v<uint32_t, RVE_N(32, 4, 1)> vuint32m4_t;
typedef rve_v<uint32_t, RVE_N(32, 8, 1)> vuint32m8_t;
typedef rve_v<uint64_t, RVE_N(64, 1, 1)> vuint64m1_t;
typedef rve_v<uint64_t, RVE_N(64, 2, 1)> vuint64m2_t;
typedef rve_v<uint64_t, RVE_N(64, 4, 1)> vuint64m4_t;
typedef rve_v<uint64_t, RVE_N(64, 8, 1)> vuint64m8_t;
typedef rve_v<uint16_t, RVE_N(16, 1, 4)> vuint16mf4_t;
typedef rve_v<uint16_t, RVE_N(16, 1, 2)> vuint16mf2_t;
typedef rve_v<uint16_t, RVE_N(16, 1, 1)> vuint16m1_t;
typedef rve_v<uint8_t, RVE_N(8, 1, 1)> vuint8m1_t;
typedef rve_b<(size_t)(RVV_EMUL_VLEN) / 4> vbool4_t;
typedef rve_b<(size_t)(RVV_EMUL_VLEN) / 8> vbool8_t;
typedef rve_b<(size_t)(RVV_EMUL_VLEN) / 16> vbool16_t;
typedef rve_b<(size_t)(RVV_EMUL_VLEN) / 32> vbool32_t;
typedef rve_b<(size_t)(RVV_EMUL_VLEN) / 64> vbool64_t;

// ------------------------------------------------------------------ vsetvl
#define RVE_SETVL(E, SEW, NUM, DEN)                                                           \
  static inline size_t __riscv_vsetvlmax_##E() { return RVE_N(SEW, NUM, DEN); }               \
  static inline size_t __riscv_vsetvl_##E(size_t avl) {                                       \
    return avl < RVE_N(SEW, NUM, DEN) ? avl : RVE_N(SEW, NUM, DEN);                           \
  }
RVE_SETVL(e8m1, 8, 1, 1)
RVE_SETVL(e16m1, 16, 1, 1)
RVE_SETVL(e32m1, 32, 1, 1)
RVE_SETVL(e32m2, 32, 2, 1)
RVE_SETVL(e32m4, 32, 4, 1)
RVE_SETVL(e32m8, 32, 8, 1)
RVE_SETVL(e64m1, 64, 1, 1)
RVE_SETVL(e64m2, 64, 2, 1)
RVE_SETVL(e64m4, 64, 4, 1)
RVE_SETVL(e64m8, 64, 8, 1)

// ------------------------------------------------- unit-stride load/store
#define RVE_LOAD(EEW, S, V, T)                                                                \
  static inline V __riscv_vle##EEW##_v_##S(const T* base, size_t vl) {                        \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = base[i];                                         \
    return r;                                                                                 \
  }
#define RVE_STORE(EEW, S, V, T)                                                               \
  static inline void __riscv_vse##EEW##_v_##S(T* base, V v, size_t vl) {                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    for (size_t i = 0; i < vl; ++i) base[i] = v.e[i];                                         \
  }

// ----------------------------------------- indexed (byte offset) load/store
#define RVE_INDEXED(S, V, T, IX, M) RVE_INDEXED_W(32, S, V, T, IX, M)
#define RVE_INDEXED_W(W, S, V, T, IX, M)                                                      \
  static inline V __riscv_vloxei##W##_v_##S(const T* base, IX bindex, size_t vl) {             \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i)                                                           \
      r.e[i] = rve::ld<T>((const char*)base + bindex.e[i]);                                   \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vloxei##W##_v_##S##_m(M mask, const T* base, IX bindex, size_t vl) {\
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i)                                                           \
      if (mask.e[i]) r.e[i] = rve::ld<T>((const char*)base + bindex.e[i]);                    \
    return r;                                                                                 \
  }                                                                                           \
  static inline void __riscv_vsoxei##W##_v_##S(T* base, IX bindex, V v, size_t vl) {           \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    for (size_t i = 0; i < vl; ++i) rve::st<T>((char*)base + bindex.e[i], v.e[i]);            \
  }                                                                                           \
  static inline void __riscv_vsoxei##W##_v_##S##_m(M mask, T* base, IX bindex, V v,           \
                                                   size_t vl) {                               \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    for (size_t i = 0; i < vl; ++i)                                                           \
      if (mask.e[i]) rve::st<T>((char*)base + bindex.e[i], v.e[i]);                           \
  }

// ------------------------------------------------------ floating point ops
#define RVE_FLOAT(S, S1, V, V1, T, M, GX)                                                     \
  static inline V __riscv_vfadd_vv_##S(V a, V b, size_t vl) {                                 \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] + b.e[i];                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfadd_vv_##S##_mu(M mask, V off, V a, V b, size_t vl) {             \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = off;                                                                                \
    for (size_t i = 0; i < vl; ++i)                                                           \
      if (mask.e[i]) r.e[i] = a.e[i] + b.e[i];                                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfsub_vv_##S(V a, V b, size_t vl) {                                 \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] - b.e[i];                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfmul_vv_##S(V a, V b, size_t vl) {                                 \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] * b.e[i];                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfmul_vf_##S(V a, T s, size_t vl) {                                 \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] * s;                                      \
    return r;                                                                                 \
  }                                                                                           \
  /* vd + vs1 * vs2 */                                                                        \
  static inline V __riscv_vfmacc_vv_##S(V vd, V vs1, V vs2, size_t vl) {                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vd;                                                                                 \
    for (size_t i = 0; i < vl; ++i) r.e[i] = std::fma(vs1.e[i], vs2.e[i], vd.e[i]);           \
    return r;                                                                                 \
  }                                                                                           \
  /* tail undisturbed: elements past vl keep vd (as the plain form does here) */              \
  static inline V __riscv_vfmacc_vv_##S##_tu(V vd, V vs1, V vs2, size_t vl) {                 \
    return __riscv_vfmacc_vv_##S(vd, vs1, vs2, vl);                                           \
  }                                                                                           \
  static inline V __riscv_vfmacc_vf_##S(V vd, T rs1, V vs2, size_t vl) {                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vd;                                                                                 \
    for (size_t i = 0; i < vl; ++i) r.e[i] = std::fma(rs1, vs2.e[i], vd.e[i]);                \
    return r;                                                                                 \
  }                                                                                           \
  /* vd * vs1 + vs2 */                                                                        \
  static inline V __riscv_vfmadd_vv_##S(V vd, V vs1, V vs2, size_t vl) {                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vd;                                                                                 \
    for (size_t i = 0; i < vl; ++i) r.e[i] = std::fma(vs1.e[i], vd.e[i], vs2.e[i]);           \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfmadd_vf_##S(V vd, T rs1, V vs2, size_t vl) {                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vd;                                                                                 \
    for (size_t i = 0; i < vl; ++i) r.e[i] = std::fma(rs1, vd.e[i], vs2.e[i]);                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V1 __riscv_vfredusum_vs_##S##_##S1(V v, V1 s, size_t vl) {                    \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V1 r = s;                                                                                 \
    T acc = s.e[0];                                                                           \
    for (size_t i = 0; i < vl; ++i) acc += v.e[i];                                            \
    if (vl) r.e[0] = acc;                                                                     \
    return r;                                                                                 \
  }                                                                                           \
  static inline V1 __riscv_vfredosum_vs_##S##_##S1(V v, V1 s, size_t vl) {                    \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V1 r = s;                                                                                 \
    T acc = s.e[0];                                                                           \
    for (size_t i = 0; i < vl; ++i) acc += v.e[i];                                            \
    if (vl) r.e[0] = acc;                                                                     \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfmv_v_f_##S(T s, size_t vl) {                                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = s;                                               \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfmv_s_f_##S##_tu(V vd, T s, size_t vl) {                           \
    V r = vd;                                                                                 \
    if (vl) r.e[0] = s;                                                                       \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfmerge_vfm_##S(V vs2, T rs1, M v0, size_t vl) {                    \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vs2;                                                                                \
    for (size_t i = 0; i < vl; ++i) r.e[i] = v0.e[i] ? rs1 : vs2.e[i];                        \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vmerge_vvm_##S(V vs2, V vs1, M v0, size_t vl) {                     \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vs2;                                                                                \
    for (size_t i = 0; i < vl; ++i) r.e[i] = v0.e[i] ? vs1.e[i] : vs2.e[i];                   \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vfslide1down_vf_##S(V vs2, T rs1, size_t vl) {                      \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vs2;                                                                                \
    for (size_t i = 0; i + 1 < vl; ++i) r.e[i] = vs2.e[i + 1];                                \
    if (vl) r.e[vl - 1] = rs1;                                                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vslideup_vx_##S(V vd, V vs2, size_t off, size_t vl) {               \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vd;                                                                                 \
    for (size_t i = off; i < vl; ++i) r.e[i] = vs2.e[i - off];                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vrgather_vv_##S(V vs2, GX idx, size_t vl) {                         \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vs2;                                                                                \
    for (size_t i = 0; i < vl; ++i)                                                           \
      r.e[i] = (size_t)idx.e[i] < rve::lanes<V>() ? vs2.e[idx.e[i]] : (T)0;                   \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vrgather_vx_##S##_mu(M mask, V off, V vs2, size_t k, size_t vl) {   \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = off;                                                                                \
    for (size_t i = 0; i < vl; ++i)                                                           \
      if (mask.e[i]) r.e[i] = k < rve::lanes<V>() ? vs2.e[k] : (T)0;                          \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vmv_v_v_##S(V v, size_t vl) {                                       \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = v.e[i];                                          \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vcompress_vm_##S(V vs2, M m, size_t vl) {                           \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = vs2;                                                                                \
    size_t k = 0;                                                                             \
    for (size_t i = 0; i < vl; ++i)                                                           \
      if (m.e[i]) r.e[k++] = vs2.e[i];                                                        \
    return r;                                                                                 \
  }                                                                                           \
  static inline T __riscv_vfmv_f_s_##S##_##T(V v) { return v.e[0]; }

// ---------------------------------------------------------- integer ops
#define RVE_UINT(S, V, T, M)                                                                  \
  static inline V __riscv_vadd_vv_##S(V a, V b, size_t vl) {                                  \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (T)(a.e[i] + b.e[i]);                            \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vadd_vx_##S##_mu(M mask, V off, V a, T s, size_t vl) {              \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = off;                                                                                \
    for (size_t i = 0; i < vl; ++i)                                                           \
      if (mask.e[i]) r.e[i] = (T)(a.e[i] + s);                                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vand_vx_##S(V a, T s, size_t vl) {                                  \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (T)(a.e[i] & s);                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vmul_vx_##S(V a, T s, size_t vl) {                                  \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (T)(a.e[i] * s);                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vsll_vx_##S(V a, size_t sh, size_t vl) {                            \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    const unsigned k = (unsigned)(sh & (8 * sizeof(T) - 1));                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (T)(a.e[i] << k);                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vsrl_vx_##S(V a, size_t sh, size_t vl) {                            \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r = a;                                                                                  \
    const unsigned k = (unsigned)(sh & (8 * sizeof(T) - 1));                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (T)(a.e[i] >> k);                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline V __riscv_vmv_v_x_##S(T s, size_t vl) {                                       \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = s;                                               \
    return r;                                                                                 \
  }                                                                                           \
  /* element i = number of set mask elements below i */                                       \
  static inline V __riscv_viota_m_##S(M m, size_t vl) {                                       \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    V r{};                                                                                    \
    T c = 0;                                                                                  \
    for (size_t i = 0; i < vl; ++i) {                                                         \
      r.e[i] = c;                                                                             \
      c = (T)(c + (m.e[i] ? 1 : 0));                                                          \
    }                                                                                         \
    return r;                                                                                 \
  }

#define RVE_UCMP(S, B, V, T, M)                                                               \
  static inline M __riscv_vmseq_vx_##S##_##B(V a, T s, size_t vl) {                           \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    M r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] == s;                                     \
    return r;                                                                                 \
  }                                                                                           \
  static inline M __riscv_vmsleu_vv_##S##_##B(V a, V b, size_t vl) {                          \
    vl = rve::avl(vl, rve::lanes<V>());                                                       \
    M r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] <= b.e[i];                                \
    return r;                                                                                 \
  }

// ----------------------------------------------------------- mask ops
#define RVE_MASK(B, M)                                                                        \
  static inline M __riscv_vmset_m_##B(size_t vl) {                                            \
    vl = rve::avl(vl, rve::lanes<M>());                                                       \
    M r{};                                                                                    \
    for (size_t i = 0; i < vl; ++i) r.e[i] = 1;                                               \
    return r;                                                                                 \
  }                                                                                           \
  static inline M __riscv_vmand_mm_##B(M a, M b, size_t vl) {                                 \
    vl = rve::avl(vl, rve::lanes<M>());                                                       \
    M r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] & b.e[i];                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline M __riscv_vmandn_mm_##B(M a, M b, size_t vl) {                                \
    vl = rve::avl(vl, rve::lanes<M>());                                                       \
    M r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] & (uint8_t)!b.e[i];                       \
    return r;                                                                                 \
  }                                                                                           \
  static inline M __riscv_vmor_mm_##B(M a, M b, size_t vl) {                                  \
    vl = rve::avl(vl, rve::lanes<M>());                                                       \
    M r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = a.e[i] | b.e[i];                                 \
    return r;                                                                                 \
  }                                                                                           \
  static inline M __riscv_vmnot_m_##B(M a, size_t vl) {                                       \
    vl = rve::avl(vl, rve::lanes<M>());                                                       \
    M r = a;                                                                                  \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (uint8_t)!a.e[i];                                \
    return r;                                                                                 \
  }                                                                                           \
  static inline unsigned long __riscv_vcpop_m_##B(M a, size_t vl) {                           \
    vl = rve::avl(vl, rve::lanes<M>());                                                       \
    unsigned long c = 0;                                                                      \
    for (size_t i = 0; i < vl; ++i) c += a.e[i] ? 1 : 0;                                      \
    return c;                                                                                 \
  }

// mask element i = bit i of the register image of the integer vector
#define RVE_REINTERPRET(S, V, B, M)                                                           \
  static inline M __riscv_vreinterpret_v_##S##_##B(V v) {                                     \
    unsigned char bytes[sizeof(v.e)];                                                         \
    std::memcpy(bytes, v.e, sizeof(v.e));                                                     \
    M r{};                                                                                    \
    for (size_t i = 0; i < rve::lanes<M>(); ++i) r.e[i] = (bytes[i / 8] >> (i % 8)) & 1u;     \
    return r;                                                                                 \
  }

// zero-extending widen u32 -> u64
#define RVE_WIDEN(S, VD, VS)                                                                  \
  static inline VD __riscv_vwcvtu_x_x_v_##S(VS v, size_t vl) {                                \
    vl = rve::avl(vl, rve::lanes<VD>());                                                      \
    VD r{};                                                                                   \
    for (size_t i = 0; i < vl; ++i) r.e[i] = (uint64_t)v.e[i];                                \
    return r;                                                                                 \
  }

// ------------------------------------------------------ instantiations
typedef double f64;
typedef float f32;
RVE_LOAD(64, f64m1, vfloat64m1_t, double)
RVE_LOAD(64, f64m2, vfloat64m2_t, double)
RVE_LOAD(64, f64m4, vfloat64m4_t, double)
RVE_LOAD(64, f64m8, vfloat64m8_t, double)
RVE_LOAD(32, f32m1, vfloat32m1_t, float)
RVE_LOAD(32, f32m2, vfloat32m2_t, float)
RVE_LOAD(32, f32m4, vfloat32m4_t, float)
RVE_LOAD(32, f32m8, vfloat32m8_t, float)
RVE_LOAD(32, u32mf2, vuint32mf2_t, uint32_t)
RVE_LOAD(32, u32m1, vuint32m1_t, uint32_t)
RVE_LOAD(32, u32m2, vuint32m2_t, uint32_t)
RVE_LOAD(32, u32m4, vuint32m4_t, uint32_t)
RVE_LOAD(32, u32m8, vuint32m8_t, uint32_t)
RVE_LOAD(16, u16mf4, vuint16mf4_t, uint16_t)
RVE_LOAD(16, u16mf2, vuint16mf2_t, uint16_t)
RVE_LOAD(16, u16m1, vuint16m1_t, uint16_t)
RVE_LOAD(8, u8m1, vuint8m1_t, uint8_t)
RVE_STORE(64, f64m1, vfloat64m1_t, double)
RVE_STORE(64, f64m2, vfloat64m2_t, double)
RVE_STORE(64, f64m4, vfloat64m4_t, double)
RVE_STORE(64, f64m8, vfloat64m8_t, double)
RVE_STORE(32, f32m1, vfloat32m1_t, float)
RVE_STORE(32, f32m2, vfloat32m2_t, float)
RVE_STORE(32, f32m4, vfloat32m4_t, float)
RVE_STORE(32, f32m8, vfloat32m8_t, float)

// index vector of EEW 32 for data of SEW: EMUL = LMUL * 32 / SEW
RVE_INDEXED(f64m1, vfloat64m1_t, double, vuint32mf2_t, vbool64_t)
RVE_INDEXED(f64m2, vfloat64m2_t, double, vuint32m1_t, vbool32_t)
RVE_INDEXED(f64m4, vfloat64m4_t, double, vuint32m2_t, vbool16_t)
RVE_INDEXED(f64m8, vfloat64m8_t, double, vuint32m4_t, vbool8_t)
RVE_INDEXED(f32m1, vfloat32m1_t, float, vuint32m1_t, vbool32_t)
RVE_INDEXED(f32m2, vfloat32m2_t, float, vuint32m2_t, vbool16_t)
RVE_INDEXED(f32m4, vfloat32m4_t, float, vuint32m4_t, vbool8_t)
RVE_INDEXED(f32m8, vfloat32m8_t, float, vuint32m8_t, vbool4_t)
RVE_INDEXED(u32mf2, vuint32mf2_t, uint32_t, vuint32mf2_t, vbool64_t)
RVE_INDEXED(u32m1, vuint32m1_t, uint32_t, vuint32m1_t, vbool32_t)
RVE_INDEXED(u32m2, vuint32m2_t, uint32_t, vuint32m2_t, vbool16_t)
RVE_INDEXED(u32m4, vuint32m4_t, uint32_t, vuint32m4_t, vbool8_t)
RVE_INDEXED(u32m8, vuint32m8_t, uint32_t, vuint32m8_t, vbool4_t)

// index vector of EEW 16 (HCSR's uint16 block columns): EMUL = LMUL * 16 / SEW
RVE_INDEXED_W(16, f64m1, vfloat64m1_t, double, vuint16mf4_t, vbool64_t)
RVE_INDEXED_W(16, f32m1, vfloat32m1_t, float, vuint16mf2_t, vbool32_t)

// gather index: same SEW, same LMUL
RVE_FLOAT(f64m1, f64m1, vfloat64m1_t, vfloat64m1_t, f64, vbool64_t, vuint64m1_t)
RVE_FLOAT(f64m2, f64m1, vfloat64m2_t, vfloat64m1_t, f64, vbool32_t, vuint64m2_t)
RVE_FLOAT(f64m4, f64m1, vfloat64m4_t, vfloat64m1_t, f64, vbool16_t, vuint64m4_t)
RVE_FLOAT(f64m8, f64m1, vfloat64m8_t, vfloat64m1_t, f64, vbool8_t, vuint64m8_t)
RVE_FLOAT(f32m1, f32m1, vfloat32m1_t, vfloat32m1_t, f32, vbool32_t, vuint32m1_t)
RVE_FLOAT(f32m2, f32m1, vfloat32m2_t, vfloat32m1_t, f32, vbool16_t, vuint32m2_t)
RVE_FLOAT(f32m4, f32m1, vfloat32m4_t, vfloat32m1_t, f32, vbool8_t, vuint32m4_t)
RVE_FLOAT(f32m8, f32m1, vfloat32m8_t, vfloat32m1_t, f32, vbool4_t, vuint32m8_t)

RVE_UINT(u16mf4, vuint16mf4_t, uint16_t, vbool64_t)
RVE_UINT(u16mf2, vuint16mf2_t, uint16_t, vbool32_t)
RVE_UINT(u32mf2, vuint32mf2_t, uint32_t, vbool64_t)
RVE_UINT(u32m1, vuint32m1_t, uint32_t, vbool32_t)
RVE_UINT(u32m2, vuint32m2_t, uint32_t, vbool16_t)
RVE_UINT(u32m4, vuint32m4_t, uint32_t, vbool8_t)
RVE_UINT(u32m8, vuint32m8_t, uint32_t, vbool4_t)
RVE_UCMP(u32mf2, b64, vuint32mf2_t, uint32_t, vbool64_t)
RVE_UCMP(u32m1, b32, vuint32m1_t, uint32_t, vbool32_t)
RVE_UCMP(u32m2, b16, vuint32m2_t, uint32_t, vbool16_t)
RVE_UCMP(u32m4, b8, vuint32m4_t, uint32_t, vbool8_t)
RVE_UCMP(u32m8, b4, vuint32m8_t, uint32_t, vbool4_t)

RVE_MASK(b4, vbool4_t)
RVE_MASK(b8, vbool8_t)
RVE_MASK(b16, vbool16_t)
RVE_MASK(b32, vbool32_t)
RVE_MASK(b64, vbool64_t)

RVE_REINTERPRET(u16m1, vuint16m1_t, b16, vbool16_t)
RVE_REINTERPRET(u8m1, vuint8m1_t, b32, vbool32_t)

RVE_WIDEN(u64m1, vuint64m1_t, vuint32mf2_t)
RVE_WIDEN(u64m2, vuint64m2_t, vuint32m1_t)
RVE_WIDEN(u64m4, vuint64m4_t, vuint32m2_t)
RVE_WIDEN(u64m8, vuint64m8_t, vuint32m4_t)
