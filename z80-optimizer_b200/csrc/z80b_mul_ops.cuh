// z80b_mul_ops.cuh -- the constant-multiply instruction model on four
// inputs per 32-bit word (one input per byte, the carry in bit 0 of each
// byte), shared by the search kernels and, compiled as plain C++, by the host
// tests that compare it with the oracle.
//
// Model: the carry-only MulState of cmd/mulopt/main.go:55-127 (A, B, carry
// and the shadows A', B', carry'), widened by C (and its shadow) for the
// 21-op workload pool.  No instruction of any pool reads a flag other than
// the carry, so tracking the carry alone yields the A of pkg/cpu.Exec.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define Z80B_MUL_HD __host__ __device__ __forceinline__
#else
#define Z80B_MUL_HD inline
#endif

namespace z80b {
namespace mul {
namespace ops {

constexpr uint32_t M1 = 0x01010101u;
constexpr uint32_t M7 = 0x7F7F7F7Fu;
constexpr uint32_t M8 = 0x80808080u;
constexpr uint32_t MHI = 0xFEFEFEFEu;

enum Kind : uint8_t {
  K_ADD_AA, K_ADD_AB, K_ADD_AC, K_SUB_B, K_SUB_C, K_LD_BA, K_LD_CA, K_LD_AB, K_LD_AC,
  K_ADC_AB, K_ADC_AA, K_SBC_AB, K_SBC_AA, K_SLA_A, K_SRA_A, K_SRL_A, K_RLA, K_RRA,
  K_RLCA, K_RRCA, K_NEG, K_CPL, K_OR_A, K_SCF, K_CCF, K_EX_AF, K_EXX
};

// Pools as types: kind per position, and a bit per position whose
// instruction takes 8 T-states (all others take 4).
// cmd/mulopt/main.go:25-49
struct PGo {
  static constexpr int N = 14;
  static constexpr Kind kind[N] = {K_ADD_AA, K_ADD_AB, K_SUB_B,  K_LD_BA,  K_SLA_A,  K_SRL_A, K_EX_AF,
                                   K_EXX,    K_ADC_AB, K_ADC_AA, K_SBC_AB, K_SBC_AA, K_OR_A,  K_NEG};
  static constexpr uint32_t t8 = (1u << 4) | (1u << 5) | (1u << 13);
};
// The 21-op pool of the constant-multiply workload.
struct PWide {
  static constexpr int N = 21;
  static constexpr Kind kind[N] = {K_ADD_AA, K_ADD_AB, K_SUB_B, K_LD_BA, K_SLA_A,  K_SRL_A, K_RLA,
                                   K_RRA,    K_RLCA,   K_RRCA,  K_NEG,   K_CPL,    K_OR_A,  K_SCF,
                                   K_CCF,    K_EX_AF,  K_LD_CA, K_ADD_AC, K_SUB_C, K_LD_AB, K_LD_AC};
  static constexpr uint32_t t8 = (1u << 4) | (1u << 5) | (1u << 10);
};
// cuda/z80_mulopt_fast.cu:20-51
struct PFast {
  static constexpr int N = 14;
  static constexpr Kind kind[N] = {K_ADD_AA, K_ADD_AB, K_SUB_B, K_LD_BA, K_ADC_AB, K_ADC_AA, K_SBC_AB,
                                   K_SBC_AA, K_SRL_A,  K_RLA,   K_RRA,   K_RLCA,   K_RRCA,   K_NEG};
  static constexpr uint32_t t8 = (1u << 8) | (1u << 13);
};
// cuda/z80_mulopt.cu:19-48 (RLC A / RRC A compute what RLCA / RRCA do)
struct PCuda {
  static constexpr int N = 21;
  static constexpr Kind kind[N] = {K_ADD_AA, K_ADD_AB, K_SUB_B, K_LD_BA, K_ADC_AB, K_ADC_AA, K_SBC_AB,
                                   K_SBC_AA, K_SLA_A,  K_SRA_A, K_SRL_A, K_RLA,    K_RRA,    K_RLCA,
                                   K_RRCA,   K_RLCA,   K_RRCA,  K_OR_A,  K_NEG,    K_SCF,    K_EX_AF};
  static constexpr uint32_t t8 = (1u << 8) | (1u << 9) | (1u << 10) | (1u << 15) | (1u << 16) | (1u << 18);
};

// Four inputs per word.
struct S4 {
  uint32_t a, b, c, as, bs, cs, cf, cfs;
};

// Bytewise x + y + cin (cin: bit 0 per byte); carry out to bit 0 per byte.
Z80B_MUL_HD uint32_t add8(uint32_t x, uint32_t y, uint32_t cin, uint32_t& cout) {
  const uint32_t l = (x & M7) + (y & M7) + cin;  // bit 7 of each byte = carry into bit 7
  cout = (((x & y) | ((x | y) & l)) >> 7) & M1;
  return l ^ ((x ^ y) & M8);
}
// Bytewise x - y - bin with the borrow out (the Z80 carry after SUB/SBC).
Z80B_MUL_HD uint32_t sub8(uint32_t x, uint32_t y, uint32_t bin, uint32_t& bout) {
  uint32_t c;
  const uint32_t r = add8(x, ~y, bin ^ M1, c);
  bout = c ^ M1;
  return r;
}

template <Kind K>
Z80B_MUL_HD void apply(S4& s) {
  uint32_t t;
  if constexpr (K == K_ADD_AA || K == K_SLA_A) {
    s.cf = (s.a >> 7) & M1;
    s.a = (s.a << 1) & MHI;
  } else if constexpr (K == K_ADD_AB) {
    s.a = add8(s.a, s.b, 0, s.cf);
  } else if constexpr (K == K_ADD_AC) {
    s.a = add8(s.a, s.c, 0, s.cf);
  } else if constexpr (K == K_SUB_B) {
    s.a = sub8(s.a, s.b, 0, s.cf);
  } else if constexpr (K == K_SUB_C) {
    s.a = sub8(s.a, s.c, 0, s.cf);
  } else if constexpr (K == K_LD_BA) {
    s.b = s.a;
  } else if constexpr (K == K_LD_CA) {
    s.c = s.a;
  } else if constexpr (K == K_LD_AB) {
    s.a = s.b;
  } else if constexpr (K == K_LD_AC) {
    s.a = s.c;
  } else if constexpr (K == K_ADC_AB) {
    s.a = add8(s.a, s.b, s.cf, s.cf);
  } else if constexpr (K == K_ADC_AA) {
    t = (s.a >> 7) & M1;
    s.a = ((s.a << 1) & MHI) | s.cf;
    s.cf = t;
  } else if constexpr (K == K_SBC_AB) {
    s.a = sub8(s.a, s.b, s.cf, s.cf);
  } else if constexpr (K == K_SBC_AA) {
    s.a = s.cf * 0xFFu;  // 0 - carry per byte; the carry stays
  } else if constexpr (K == K_SRA_A) {
    s.cf = s.a & M1;
    s.a = ((s.a >> 1) & M7) | (s.a & M8);
  } else if constexpr (K == K_SRL_A) {
    s.cf = s.a & M1;
    s.a = (s.a >> 1) & M7;
  } else if constexpr (K == K_RLA) {
    t = (s.a >> 7) & M1;
    s.a = ((s.a << 1) & MHI) | s.cf;
    s.cf = t;
  } else if constexpr (K == K_RRA) {
    t = s.a & M1;
    s.a = ((s.a >> 1) & M7) | (s.cf << 7);
    s.cf = t;
  } else if constexpr (K == K_RLCA) {
    s.cf = (s.a >> 7) & M1;
    s.a = ((s.a << 1) & MHI) | s.cf;
  } else if constexpr (K == K_RRCA) {
    s.cf = s.a & M1;
    s.a = ((s.a >> 1) & M7) | (s.cf << 7);
  } else if constexpr (K == K_NEG) {
    s.a = sub8(0u, s.a, 0u, s.cf);
  } else if constexpr (K == K_CPL) {
    s.a = ~s.a;
  } else if constexpr (K == K_OR_A) {
    s.cf = 0;
  } else if constexpr (K == K_SCF) {
    s.cf = M1;
  } else if constexpr (K == K_CCF) {
    s.cf ^= M1;
  } else if constexpr (K == K_EX_AF) {
    t = s.a; s.a = s.as; s.as = t;
    t = s.cf; s.cf = s.cfs; s.cfs = t;
  } else if constexpr (K == K_EXX) {
    t = s.b; s.b = s.bs; s.bs = t;
    t = s.c; s.c = s.cs; s.cs = t;
  }
}

// Instruction i of pool P (i warp-uniform at every call site).
template <class P>
Z80B_MUL_HD void apply_at(int i, S4& s) {
  switch (i) {
#define Z80B_MUL_CASE(j) \
  case j:                \
    if constexpr (j < P::N) apply<P::kind[j]>(s); \
    break;
    Z80B_MUL_CASE(0) Z80B_MUL_CASE(1) Z80B_MUL_CASE(2) Z80B_MUL_CASE(3) Z80B_MUL_CASE(4)
    Z80B_MUL_CASE(5) Z80B_MUL_CASE(6) Z80B_MUL_CASE(7) Z80B_MUL_CASE(8) Z80B_MUL_CASE(9)
    Z80B_MUL_CASE(10) Z80B_MUL_CASE(11) Z80B_MUL_CASE(12) Z80B_MUL_CASE(13) Z80B_MUL_CASE(14)
    Z80B_MUL_CASE(15) Z80B_MUL_CASE(16) Z80B_MUL_CASE(17) Z80B_MUL_CASE(18) Z80B_MUL_CASE(19)
    Z80B_MUL_CASE(20)
#undef Z80B_MUL_CASE
    default: break;
  }
}

template <class P>
Z80B_MUL_HD uint32_t cost_of(int i) {
  return 4u + 4u * ((P::t8 >> i) & 1u);
}

}  // namespace ops
}  // namespace mul
}  // namespace z80b
