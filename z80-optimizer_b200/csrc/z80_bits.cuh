// z80_bits.cuh -- bit-sliced Z80 step: 32 states at once, one 32-bit word
// per register bit ("plane"), bit j of every plane belonging to state j.
//
// Every instruction becomes word-wide logic on planes: an 8-bit add is a
// ripple of 8 majority/xor steps for all 32 states, a register move is a
// copy of 8 words, a flag is one plane.  The results follow the scalar step
// function of z80_exec.cuh bit for bit (pkg/cpu/exec.go semantics, flag
// formulas included); the host tests compare the two on every opcode.  The
// ExhaustiveCheck sweep uses it for A-blocks: a lane holds 32 consecutive
// values of A with the other registers equal across them.
#pragma once
#include <cstdint>

#include "z80_exec.cuh"

namespace z80b {

struct ZB {
  uint32_t a[8], f[8], b[8], c[8], d[8], e[8], h[8], l[8], m[8];
  uint32_t sp[16];
};
// A compact state for pairs whose instructions name no register but B and C
// (after renaming) and neither SP nor the memory byte: D, E, H, L and M
// share one scratch array that such instructions never touch, SP another.
// The step functions below are templates over the state type.
struct ZBc {
  uint32_t a[8], f[8], b[8], c[8];
  union {
    uint32_t x[8], d[8], e[8], h[8], l[8], m[8];
  };
  uint32_t sp[16];
};

constexpr uint32_t kZBOnes = 0xFFFFFFFFu;

#if defined(__CUDA_ARCH__)  // device pass only: host compilers do not know the pragma
#define ZB_UNROLL _Pragma("unroll")
#else
#define ZB_UNROLL
#endif

Z80_HD uint32_t zb_maj(uint32_t x, uint32_t y, uint32_t z) { return (x & y) | (z & (x | y)); }
Z80_HD uint32_t zb_any(const uint32_t (&r)[8]) {
  return (r[0] | r[1] | r[2] | r[3]) | (r[4] | r[5] | r[6] | r[7]);
}
// P/V after logic ops: set when the number of one bits is even.
Z80_HD uint32_t zb_even(const uint32_t (&r)[8]) {
  return ~((r[0] ^ r[1] ^ r[2] ^ r[3]) ^ (r[4] ^ r[5] ^ r[6] ^ r[7]));
}
Z80_HD void zb_set8(uint32_t (&r)[8], uint32_t v) {
  ZB_UNROLL for (int i = 0; i < 8; i++) r[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
}
Z80_HD void zb_copy8(uint32_t (&d)[8], const uint32_t (&s)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) d[i] = s[i];
}
// S, Z, 5, 3 of a result (z_sz53), P/V and H, N cleared.
template <class ZT>
Z80_HD void zb_sz53p(ZT& z, const uint32_t (&r)[8], uint32_t carry) {
  z.f[0] = carry;
  z.f[1] = 0;
  z.f[2] = zb_even(r);
  z.f[3] = r[3];
  z.f[4] = 0;
  z.f[5] = r[5];
  z.f[6] = ~zb_any(r);
  z.f[7] = r[7];
}

// ---- 8-bit ALU (z_add .. z_cp)
// r = x + y + cin; *c4 = carry into bit 4; returns the carry out.
Z80_HD uint32_t zb_adder8(const uint32_t (&x)[8], const uint32_t (&y)[8], uint32_t cin, uint32_t (&r)[8],
                          uint32_t* c4) {
  uint32_t c = cin;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    if (i == 4) *c4 = c;
    r[i] = x[i] ^ y[i] ^ c;
    c = zb_maj(x[i], y[i], c);
  }
  return c;
}
template <class ZT>
Z80_HD void zb_add(ZT& z, const uint32_t (&v)[8], uint32_t cin) {
  uint32_t r[8], c4 = 0;
  const uint32_t co = zb_adder8(z.a, v, cin, r, &c4);
  z.f[0] = co;
  z.f[1] = 0;
  z.f[2] = (z.a[7] ^ r[7]) & (v[7] ^ r[7]);
  z.f[3] = r[3];
  z.f[4] = c4;
  z.f[5] = r[5];
  z.f[6] = ~zb_any(r);
  z.f[7] = r[7];
  zb_copy8(z.a, r);
}
// x - v - bin: the adder on ~v with carry in ~bin; the carry out is ~borrow.
Z80_HD uint32_t zb_suber8(const uint32_t (&x)[8], const uint32_t (&v)[8], uint32_t bin, uint32_t (&r)[8],
                          uint32_t* h) {
  uint32_t nv[8];
  ZB_UNROLL for (int i = 0; i < 8; i++) nv[i] = ~v[i];
  uint32_t c4 = 0;
  const uint32_t co = zb_adder8(x, nv, ~bin, r, &c4);
  *h = ~c4;  // bit 4 of x ^ v ^ r
  return ~co;
}
template <class ZT>
Z80_HD void zb_sub(ZT& z, const uint32_t (&v)[8], uint32_t bin) {
  uint32_t r[8], h = 0;
  const uint32_t borrow = zb_suber8(z.a, v, bin, r, &h);
  z.f[0] = borrow;
  z.f[1] = kZBOnes;
  z.f[2] = (z.a[7] ^ v[7]) & (z.a[7] ^ r[7]);
  z.f[3] = r[3];
  z.f[4] = h;
  z.f[5] = r[5];
  z.f[6] = ~zb_any(r);
  z.f[7] = r[7];
  zb_copy8(z.a, r);
}
template <class ZT>
Z80_HD void zb_cp(ZT& z, const uint32_t (&v)[8]) {
  uint32_t r[8], h = 0;
  const uint32_t borrow = zb_suber8(z.a, v, 0u, r, &h);
  z.f[0] = borrow;
  z.f[1] = kZBOnes;
  z.f[2] = (z.a[7] ^ v[7]) & (z.a[7] ^ r[7]);
  z.f[3] = v[3];
  z.f[4] = h;
  z.f[5] = v[5];
  z.f[6] = ~zb_any(r);
  z.f[7] = r[7];
}
template <class ZT>
Z80_HD void zb_and(ZT& z, const uint32_t (&v)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) z.a[i] &= v[i];
  zb_sz53p(z, z.a, 0u);
  z.f[4] = kZBOnes;
}
template <class ZT>
Z80_HD void zb_xor(ZT& z, const uint32_t (&v)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) z.a[i] ^= v[i];
  zb_sz53p(z, z.a, 0u);
}
template <class ZT>
Z80_HD void zb_or(ZT& z, const uint32_t (&v)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) z.a[i] |= v[i];
  zb_sz53p(z, z.a, 0u);
}
// z_inc / z_dec
template <class ZT>
Z80_HD void zb_inc(ZT& z, uint32_t (&r)[8]) {
  uint32_t c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const uint32_t t = r[i];
    r[i] = t ^ c;
    c = t & c;
  }
  z.f[1] = 0;
  z.f[2] = r[7] & ~(r[0] | r[1] | r[2] | r[3] | r[4] | r[5] | r[6]);
  z.f[3] = r[3];
  z.f[4] = ~(r[0] | r[1] | r[2] | r[3]);
  z.f[5] = r[5];
  z.f[6] = ~zb_any(r);
  z.f[7] = r[7];
}
template <class ZT>
Z80_HD void zb_dec(ZT& z, uint32_t (&r)[8]) {
  z.f[4] = ~(r[0] | r[1] | r[2] | r[3]);
  uint32_t c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const uint32_t t = r[i];
    r[i] = t ^ c;
    c = ~t & c;
  }
  z.f[1] = kZBOnes;
  z.f[2] = ~r[7] & (r[0] & r[1] & r[2] & r[3] & r[4] & r[5] & r[6]);
  z.f[3] = r[3];
  z.f[5] = r[5];
  z.f[6] = ~zb_any(r);
  z.f[7] = r[7];
}
// z_daa: corrections chosen per state, the add or the subtract selected by N.
template <class ZT>
Z80_HD void zb_daa(ZT& z) {
  const uint32_t lo_gt9 = z.a[3] & (z.a[2] | z.a[1]);
  const uint32_t hi_gt9 = z.a[7] & (z.a[6] | z.a[5]);
  const uint32_t hi_eq9 = z.a[7] & ~z.a[6] & ~z.a[5] & z.a[4];
  const uint32_t gt99 = hi_gt9 | (hi_eq9 & lo_gt9);
  const uint32_t add6 = z.f[4] | lo_gt9;
  const uint32_t add60 = z.f[0] | gt99;
  const uint32_t carry = z.f[0] | gt99;
  uint32_t v[8] = {0u, add6, add6, 0u, 0u, add60, add60, 0u};
  ZT za = z, zs = z;
  zb_add(za, v, 0u);
  zb_sub(zs, v, 0u);
  const uint32_t n = z.f[1];
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    z.a[i] = (zs.a[i] & n) | (za.a[i] & ~n);
    z.f[i] = (zs.f[i] & n) | (za.f[i] & ~n);
  }
  z.f[0] = carry;
  z.f[2] = zb_even(z.a);
}
// ---- CB rotates and shifts; results into r, flags from the new value
template <class ZT>
Z80_HD void zb_rot(ZT& z, uint32_t (&r)[8], int kind) {
  uint32_t n[8], co = 0;
  switch (kind) {
    case 0:  // RLC
      co = r[7];
      n[0] = r[7];
      ZB_UNROLL for (int i = 1; i < 8; i++) n[i] = r[i - 1];
      break;
    case 1:  // RRC
      co = r[0];
      ZB_UNROLL for (int i = 0; i < 7; i++) n[i] = r[i + 1];
      n[7] = r[0];
      break;
    case 2:  // RL
      co = r[7];
      n[0] = z.f[0];
      ZB_UNROLL for (int i = 1; i < 8; i++) n[i] = r[i - 1];
      break;
    case 3:  // RR
      co = r[0];
      ZB_UNROLL for (int i = 0; i < 7; i++) n[i] = r[i + 1];
      n[7] = z.f[0];
      break;
    case 4:  // SLA
      co = r[7];
      n[0] = 0;
      ZB_UNROLL for (int i = 1; i < 8; i++) n[i] = r[i - 1];
      break;
    case 5:  // SRA
      co = r[0];
      ZB_UNROLL for (int i = 0; i < 7; i++) n[i] = r[i + 1];
      n[7] = r[7];
      break;
    case 6:  // SRL
      co = r[0];
      ZB_UNROLL for (int i = 0; i < 7; i++) n[i] = r[i + 1];
      n[7] = 0;
      break;
    default:  // SLL
      co = r[7];
      n[0] = kZBOnes;
      ZB_UNROLL for (int i = 1; i < 8; i++) n[i] = r[i - 1];
      break;
  }
  zb_copy8(r, n);
  zb_sz53p(z, r, co);
}
template <class ZT>
Z80_HD void zb_bit(ZT& z, const uint32_t (&r)[8], int bit) {
  const uint32_t nb = ~r[bit];
  z.f[1] = 0;
  z.f[2] = nb;
  z.f[3] = r[3];
  z.f[4] = kZBOnes;
  z.f[5] = r[5];
  z.f[6] = nb;
  z.f[7] = bit == 7 ? r[7] : 0u;
}
// ---- 16-bit arithmetic on (hi, lo) register pairs
Z80_HD void zb_inc16(uint32_t (&hi)[8], uint32_t (&lo)[8], bool dec) {
  uint32_t c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const uint32_t t = lo[i];
    lo[i] = t ^ c;
    c = (dec ? ~t : t) & c;
  }
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const uint32_t t = hi[i];
    hi[i] = t ^ c;
    c = (dec ? ~t : t) & c;
  }
}
Z80_HD void zb_incsp(uint32_t (&sp)[16], bool dec) {
  uint32_t c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 16; i++) {
    const uint32_t t = sp[i];
    sp[i] = t ^ c;
    c = (dec ? ~t : t) & c;
  }
}
// HL + v (+ carry) / HL - v - carry over 16 planes, in place; kind 0 ADD,
// 1 ADC, 2 SBC.  v is given as its low and high byte planes (vlo, vhi),
// which may be HL's own: bit i of both operands is read before bit i of HL
// is written.
template <class ZT>
Z80_HD void zb_hl16(ZT& z, const uint32_t* vlo, const uint32_t* vhi, int kind) {
  uint32_t c = kind == 0 ? 0u : (kind == 1 ? z.f[0] : ~z.f[0]), c12 = 0, nz = 0, x15 = 0, v15 = 0;
  ZB_UNROLL for (int i = 0; i < 16; i++) {
    uint32_t& xr = i < 8 ? z.l[i] : z.h[i - 8];
    const uint32_t vi = i < 8 ? vlo[i] : vhi[i - 8];
    const uint32_t x = xr, y = kind == 2 ? ~vi : vi;
    if (i == 12) c12 = c;
    if (i == 15) {
      x15 = x;
      v15 = vi;
    }
    const uint32_t r = x ^ y ^ c;
    c = zb_maj(x, y, c);
    xr = r;
    nz |= r;
  }
  const uint32_t r15 = z.h[7];
  if (kind == 0) {
    z.f[0] = c;
    z.f[1] = 0;
    z.f[3] = z.h[3];
    z.f[4] = c12;
    z.f[5] = z.h[5];
    return;
  }
  if (kind == 1) {
    z.f[0] = c;
    z.f[1] = 0;
    z.f[2] = (x15 ^ r15) & (v15 ^ r15);
    z.f[4] = c12;
  } else {
    z.f[0] = ~c;
    z.f[1] = kZBOnes;
    z.f[2] = (x15 ^ v15) & (x15 ^ r15);
    z.f[4] = ~c12;
  }
  z.f[3] = z.h[3];
  z.f[5] = z.h[5];
  z.f[6] = ~nz;
  z.f[7] = r15;
}

// Register families in the enum's orders (as z80_exec.cuh's Z80B_R7 / Z80B_S7).
#define ZB_R7(M, base) M((base) + 0, a) M((base) + 1, b) M((base) + 2, c) M((base) + 3, d) \
  M((base) + 4, e) M((base) + 5, h) M((base) + 6, l)
#define ZB_S7(M, base) M((base) + 0, b) M((base) + 1, c) M((base) + 2, d) M((base) + 3, e) \
  M((base) + 4, h) M((base) + 5, l) M((base) + 6, a)

#define ZB_LDA(o, r) case (o): zb_copy8(z.a, z.r); break;
#define ZB_LDB(o, r) case (o): zb_copy8(z.b, z.r); break;
#define ZB_LDC(o, r) case (o): zb_copy8(z.c, z.r); break;
#define ZB_LDD(o, r) case (o): zb_copy8(z.d, z.r); break;
#define ZB_LDE(o, r) case (o): zb_copy8(z.e, z.r); break;
#define ZB_LDH(o, r) case (o): zb_copy8(z.h, z.r); break;
#define ZB_LDL(o, r) case (o): zb_copy8(z.l, z.r); break;
#define ZB_LDN(o, r) case (o): zb_set8(z.r, imm & 0xFFu); break;
#define ZB_ADD(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_add(z, v_, 0u); } break;
#define ZB_ADC(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_add(z, v_, z.f[0]); } break;
#define ZB_SUB(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_sub(z, v_, 0u); } break;
#define ZB_SBC(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_sub(z, v_, z.f[0]); } break;
#define ZB_AND(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_and(z, v_); } break;
#define ZB_XOR(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_xor(z, v_); } break;
#define ZB_OR(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_or(z, v_); } break;
#define ZB_CP(o, r) case (o): { uint32_t v_[8]; zb_copy8(v_, z.r); zb_cp(z, v_); } break;
#define ZB_INC(o, r) case (o): zb_inc(z, z.r); break;
#define ZB_DEC(o, r) case (o): zb_dec(z, z.r); break;
#define ZB_RLC(o, r) case (o): zb_rot(z, z.r, 0); break;
#define ZB_RRC(o, r) case (o): zb_rot(z, z.r, 1); break;
#define ZB_RL(o, r) case (o): zb_rot(z, z.r, 2); break;
#define ZB_RR(o, r) case (o): zb_rot(z, z.r, 3); break;
#define ZB_SLA(o, r) case (o): zb_rot(z, z.r, 4); break;
#define ZB_SRA(o, r) case (o): zb_rot(z, z.r, 5); break;
#define ZB_SRL(o, r) case (o): zb_rot(z, z.r, 6); break;
#define ZB_SLL(o, r) case (o): zb_rot(z, z.r, 7); break;
#define ZB_BIT(o, r) case (o): zb_bit(z, z.r, ((o) - BIT_0_A) / 7); break;
#define ZB_RES(o, r) case (o): z.r[((o) - RES_0_A) / 7] = 0u; break;
#define ZB_SET(o, r) case (o): z.r[((o) - SET_0_A) / 7] = kZBOnes; break;

// The instructions that touch only A and F (RLCA, RRCA, RLA, RRA, DAA,
// CPL, SCF, CCF, NEG, NOP); false for any other opcode.
template <class ZT>
Z80_HD bool zb_acc_step(ZT& z, uint32_t op) {
  uint32_t t8[8];
  switch (op) {
    case RLCA: {
      const uint32_t o7 = z.a[7];
      for (int i = 7; i > 0; i--) z.a[i] = z.a[i - 1];
      z.a[0] = o7;
      z.f[0] = o7; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case RRCA: {
      const uint32_t o0 = z.a[0];
      for (int i = 0; i < 7; i++) z.a[i] = z.a[i + 1];
      z.a[7] = o0;
      z.f[0] = o0; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case RLA: {
      const uint32_t o7 = z.a[7];
      for (int i = 7; i > 0; i--) z.a[i] = z.a[i - 1];
      z.a[0] = z.f[0];
      z.f[0] = o7; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case RRA: {
      const uint32_t o0 = z.a[0];
      for (int i = 0; i < 7; i++) z.a[i] = z.a[i + 1];
      z.a[7] = z.f[0];
      z.f[0] = o0; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case DAA: zb_daa(z); break;
    case CPL:
      for (int i = 0; i < 8; i++) z.a[i] = ~z.a[i];
      z.f[1] = kZBOnes; z.f[3] = z.a[3]; z.f[4] = kZBOnes; z.f[5] = z.a[5];
      break;
    case SCF: z.f[0] = kZBOnes; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5]; break;
    case CCF: z.f[4] = z.f[0]; z.f[0] = ~z.f[0]; z.f[1] = 0; z.f[3] = z.a[3]; z.f[5] = z.a[5]; break;
    case NEG: {
      zb_copy8(t8, z.a);
      zb_set8(z.a, 0u);
      zb_sub(z, t8, 0u);
    } break;
    case NOP: break;
    default: return false;
  }
  return true;
}

// The cases of the step for every instruction that names no register but
// A, F, B..L (neither SP nor the memory byte), shared by zb_step and zb6_step.
#define ZB_REG_CASES \
    ZB_S7(ZB_LDA, LD_A_B) \
    ZB_R7(ZB_LDB, LD_B_A) \
    ZB_R7(ZB_LDC, LD_C_A) \
    ZB_R7(ZB_LDD, LD_D_A) \
    ZB_R7(ZB_LDE, LD_E_A) \
    ZB_R7(ZB_LDH, LD_H_A) \
    ZB_R7(ZB_LDL, LD_L_A) \
    ZB_R7(ZB_LDN, LD_A_N) \
    ZB_S7(ZB_ADD, ADD_A_B) \
    case ADD_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, 0u); break; \
    ZB_S7(ZB_ADC, ADC_A_B) \
    case ADC_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, z.f[0]); break; \
    ZB_S7(ZB_SUB, SUB_B) \
    case SUB_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, 0u); break; \
    ZB_S7(ZB_SBC, SBC_A_B) \
    case SBC_A_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, z.f[0]); break; \
    ZB_S7(ZB_AND, AND_B) \
    case AND_N: zb_set8(t8, imm & 0xFFu); zb_and(z, t8); break; \
    ZB_S7(ZB_XOR, XOR_B) \
    case XOR_N: zb_set8(t8, imm & 0xFFu); zb_xor(z, t8); break; \
    ZB_S7(ZB_OR, OR_B) \
    case OR_N: zb_set8(t8, imm & 0xFFu); zb_or(z, t8); break; \
    ZB_S7(ZB_CP, CP_B) \
    case CP_N: zb_set8(t8, imm & 0xFFu); zb_cp(z, t8); break; \
    ZB_R7(ZB_INC, INC_A) \
    ZB_R7(ZB_DEC, DEC_A) \
    ZB_R7(ZB_RLC, RLC_A) \
    ZB_R7(ZB_RRC, RRC_A) \
    ZB_R7(ZB_RL, RL_A) \
    ZB_R7(ZB_RR, RR_A) \
    ZB_R7(ZB_SLA, SLA_A) \
    ZB_R7(ZB_SRA, SRA_A) \
    ZB_R7(ZB_SRL, SRL_A) \
    ZB_R7(ZB_SLL, SLL_A) \
    ZB_R7(ZB_BIT, BIT_0_A) ZB_R7(ZB_BIT, BIT_1_A) ZB_R7(ZB_BIT, BIT_2_A) ZB_R7(ZB_BIT, BIT_3_A) \
    ZB_R7(ZB_BIT, BIT_4_A) ZB_R7(ZB_BIT, BIT_5_A) ZB_R7(ZB_BIT, BIT_6_A) ZB_R7(ZB_BIT, BIT_7_A) \
    ZB_R7(ZB_RES, RES_0_A) ZB_R7(ZB_RES, RES_1_A) ZB_R7(ZB_RES, RES_2_A) ZB_R7(ZB_RES, RES_3_A) \
    ZB_R7(ZB_RES, RES_4_A) ZB_R7(ZB_RES, RES_5_A) ZB_R7(ZB_RES, RES_6_A) ZB_R7(ZB_RES, RES_7_A) \
    ZB_R7(ZB_SET, SET_0_A) ZB_R7(ZB_SET, SET_1_A) ZB_R7(ZB_SET, SET_2_A) ZB_R7(ZB_SET, SET_3_A) \
    ZB_R7(ZB_SET, SET_4_A) ZB_R7(ZB_SET, SET_5_A) ZB_R7(ZB_SET, SET_6_A) ZB_R7(ZB_SET, SET_7_A) \
    case INC_BC: zb_inc16(z.b, z.c, false); break; \
    case INC_DE: zb_inc16(z.d, z.e, false); break; \
    case INC_HL: zb_inc16(z.h, z.l, false); break; \
    case DEC_BC: zb_inc16(z.b, z.c, true); break; \
    case DEC_DE: zb_inc16(z.d, z.e, true); break; \
    case DEC_HL: zb_inc16(z.h, z.l, true); break; \
    case ADD_HL_BC: zb_hl16(z, z.c, z.b, 0); break; \
    case ADD_HL_DE: zb_hl16(z, z.e, z.d, 0); break; \
    case ADD_HL_HL: zb_hl16(z, z.l, z.h, 0); break; \
    case EX_DE_HL: \
      for (int i = 0; i < 8; i++) { \
        const uint32_t dd = z.d[i], ee = z.e[i]; \
        z.d[i] = z.h[i]; \
        z.e[i] = z.l[i]; \
        z.h[i] = dd; \
        z.l[i] = ee; \
      } \
      break; \
    case LD_BC_NN: zb_set8(z.b, (imm >> 8) & 0xFFu); zb_set8(z.c, imm & 0xFFu); break; \
    case LD_DE_NN: zb_set8(z.d, (imm >> 8) & 0xFFu); zb_set8(z.e, imm & 0xFFu); break; \
    case LD_HL_NN: zb_set8(z.h, (imm >> 8) & 0xFFu); zb_set8(z.l, imm & 0xFFu); break; \
    case ADC_HL_BC: zb_hl16(z, z.c, z.b, 1); break; \
    case ADC_HL_DE: zb_hl16(z, z.e, z.d, 1); break; \
    case ADC_HL_HL: zb_hl16(z, z.l, z.h, 1); break; \
    case SBC_HL_BC: zb_hl16(z, z.c, z.b, 2); break; \
    case SBC_HL_DE: zb_hl16(z, z.e, z.d, 2); break; \
    case SBC_HL_HL: zb_hl16(z, z.l, z.h, 2); break; \
  /* end of ZB_REG_CASES */

// One instruction on the 32 states of z (op and imm are the same for all).
template <class ZT>
Z80_HD void zb_step(ZT& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZB_REG_CASES
    case INC_SP: zb_incsp(z.sp, false); break;
    case DEC_SP: zb_incsp(z.sp, true); break;
    case ADD_HL_SP: zb_hl16(z, z.sp, z.sp + 8, 0); break;
    case LD_SP_HL: for (int i = 0; i < 8; i++) { z.sp[i] = z.l[i]; z.sp[i + 8] = z.h[i]; } break;
    case LD_SP_NN: for (int i = 0; i < 16; i++) z.sp[i] = ((imm >> i) & 1u) ? kZBOnes : 0u; break;
    case ADC_HL_SP: zb_hl16(z, z.sp, z.sp + 8, 1); break;
    case SBC_HL_SP: zb_hl16(z, z.sp, z.sp + 8, 2); break;
    // memory ops on the single byte M (exec.go:883-1028)
    case LD_A_HLI: zb_copy8(z.a, z.m); break;
    case LD_B_HLI: zb_copy8(z.b, z.m); break;
    case LD_C_HLI: zb_copy8(z.c, z.m); break;
    case LD_D_HLI: zb_copy8(z.d, z.m); break;
    case LD_E_HLI: zb_copy8(z.e, z.m); break;
    case LD_H_HLI: zb_copy8(z.h, z.m); break;
    case LD_L_HLI: zb_copy8(z.l, z.m); break;
    case LD_HLI_A: zb_copy8(z.m, z.a); break;
    case LD_HLI_B: zb_copy8(z.m, z.b); break;
    case LD_HLI_C: zb_copy8(z.m, z.c); break;
    case LD_HLI_D: zb_copy8(z.m, z.d); break;
    case LD_HLI_E: zb_copy8(z.m, z.e); break;
    case LD_HLI_H: zb_copy8(z.m, z.h); break;
    case LD_HLI_L: zb_copy8(z.m, z.l); break;
    case LD_HLI_N: zb_set8(z.m, imm & 0xFFu); break;
    case LD_A_BCI: case LD_A_DEI: zb_copy8(z.a, z.m); break;
    case LD_BCI_A: case LD_DEI_A: zb_copy8(z.m, z.a); break;
    case ADD_A_HLI: zb_copy8(t8, z.m); zb_add(z, t8, 0u); break;
    case ADC_A_HLI: zb_copy8(t8, z.m); zb_add(z, t8, z.f[0]); break;
    case SUB_HLI: zb_copy8(t8, z.m); zb_sub(z, t8, 0u); break;
    case SBC_A_HLI: zb_copy8(t8, z.m); zb_sub(z, t8, z.f[0]); break;
    case AND_HLI: zb_copy8(t8, z.m); zb_and(z, t8); break;
    case XOR_HLI: zb_copy8(t8, z.m); zb_xor(z, t8); break;
    case OR_HLI: zb_copy8(t8, z.m); zb_or(z, t8); break;
    case CP_HLI: zb_copy8(t8, z.m); zb_cp(z, t8); break;
    case INC_HLI: zb_inc(z, z.m); break;
    case DEC_HLI: zb_dec(z, z.m); break;
    case RLC_HLI: zb_rot(z, z.m, 0); break;
    case RRC_HLI: zb_rot(z, z.m, 1); break;
    case RL_HLI: zb_rot(z, z.m, 2); break;
    case RR_HLI: zb_rot(z, z.m, 3); break;
    case SLA_HLI: zb_rot(z, z.m, 4); break;
    case SRA_HLI: zb_rot(z, z.m, 5); break;
    case SRL_HLI: zb_rot(z, z.m, 6); break;
    case SLL_HLI: zb_rot(z, z.m, 7); break;
    case BIT_0_HLI: zb_bit(z, z.m, 0); break;
    case BIT_1_HLI: zb_bit(z, z.m, 1); break;
    case BIT_2_HLI: zb_bit(z, z.m, 2); break;
    case BIT_3_HLI: zb_bit(z, z.m, 3); break;
    case BIT_4_HLI: zb_bit(z, z.m, 4); break;
    case BIT_5_HLI: zb_bit(z, z.m, 5); break;
    case BIT_6_HLI: zb_bit(z, z.m, 6); break;
    case BIT_7_HLI: zb_bit(z, z.m, 7); break;
    case RES_0_HLI: z.m[0] = 0u; break;
    case RES_1_HLI: z.m[1] = 0u; break;
    case RES_2_HLI: z.m[2] = 0u; break;
    case RES_3_HLI: z.m[3] = 0u; break;
    case RES_4_HLI: z.m[4] = 0u; break;
    case RES_5_HLI: z.m[5] = 0u; break;
    case RES_6_HLI: z.m[6] = 0u; break;
    case RES_7_HLI: z.m[7] = 0u; break;
    case SET_0_HLI: z.m[0] = kZBOnes; break;
    case SET_1_HLI: z.m[1] = kZBOnes; break;
    case SET_2_HLI: z.m[2] = kZBOnes; break;
    case SET_3_HLI: z.m[3] = kZBOnes; break;
    case SET_4_HLI: z.m[4] = kZBOnes; break;
    case SET_5_HLI: z.m[5] = kZBOnes; break;
    case SET_6_HLI: z.m[6] = kZBOnes; break;
    case SET_7_HLI: z.m[7] = kZBOnes; break;
    default: zb_acc_step(z, op); break;
  }
}

// The A, F, B, C state of a compact sweep.  A compact program (a pair's
// instructions renamed by compact_map) names no register but A, F, B and C
// and neither SP nor the memory byte, so nothing else needs to be held.
struct ZB4 {
  uint32_t a[8], f[8], b[8], c[8];
};
#define ZB4_R(M, base) M((base) + 0, a) M((base) + 1, b) M((base) + 2, c)
#define ZB4_S(M, base) M((base) + 0, b) M((base) + 1, c) M((base) + 6, a)

// The step on ZB4: the cases of zb_step for every instruction that names no
// register but A, F, B and C (the only ones a compact program holds); any
// other opcode leaves the state unchanged and must not occur.
Z80_HD void zb4_step(ZB4& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZB4_S(ZB_LDA, LD_A_B)
    ZB4_R(ZB_LDB, LD_B_A)
    ZB4_R(ZB_LDC, LD_C_A)
    ZB4_R(ZB_LDN, LD_A_N)
    ZB4_S(ZB_ADD, ADD_A_B)
    case ADD_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, 0u); break;
    ZB4_S(ZB_ADC, ADC_A_B)
    case ADC_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, z.f[0]); break;
    ZB4_S(ZB_SUB, SUB_B)
    case SUB_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, 0u); break;
    ZB4_S(ZB_SBC, SBC_A_B)
    case SBC_A_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, z.f[0]); break;
    ZB4_S(ZB_AND, AND_B)
    case AND_N: zb_set8(t8, imm & 0xFFu); zb_and(z, t8); break;
    ZB4_S(ZB_XOR, XOR_B)
    case XOR_N: zb_set8(t8, imm & 0xFFu); zb_xor(z, t8); break;
    ZB4_S(ZB_OR, OR_B)
    case OR_N: zb_set8(t8, imm & 0xFFu); zb_or(z, t8); break;
    ZB4_S(ZB_CP, CP_B)
    case CP_N: zb_set8(t8, imm & 0xFFu); zb_cp(z, t8); break;
    ZB4_R(ZB_INC, INC_A)
    ZB4_R(ZB_DEC, DEC_A)
    ZB4_R(ZB_RLC, RLC_A)
    ZB4_R(ZB_RRC, RRC_A)
    ZB4_R(ZB_RL, RL_A)
    ZB4_R(ZB_RR, RR_A)
    ZB4_R(ZB_SLA, SLA_A)
    ZB4_R(ZB_SRA, SRA_A)
    ZB4_R(ZB_SRL, SRL_A)
    ZB4_R(ZB_SLL, SLL_A)
    ZB4_R(ZB_BIT, BIT_0_A) ZB4_R(ZB_BIT, BIT_1_A) ZB4_R(ZB_BIT, BIT_2_A) ZB4_R(ZB_BIT, BIT_3_A)
    ZB4_R(ZB_BIT, BIT_4_A) ZB4_R(ZB_BIT, BIT_5_A) ZB4_R(ZB_BIT, BIT_6_A) ZB4_R(ZB_BIT, BIT_7_A)
    ZB4_R(ZB_RES, RES_0_A) ZB4_R(ZB_RES, RES_1_A) ZB4_R(ZB_RES, RES_2_A) ZB4_R(ZB_RES, RES_3_A)
    ZB4_R(ZB_RES, RES_4_A) ZB4_R(ZB_RES, RES_5_A) ZB4_R(ZB_RES, RES_6_A) ZB4_R(ZB_RES, RES_7_A)
    ZB4_R(ZB_SET, SET_0_A) ZB4_R(ZB_SET, SET_1_A) ZB4_R(ZB_SET, SET_2_A) ZB4_R(ZB_SET, SET_3_A)
    ZB4_R(ZB_SET, SET_4_A) ZB4_R(ZB_SET, SET_5_A) ZB4_R(ZB_SET, SET_6_A) ZB4_R(ZB_SET, SET_7_A)
    case INC_BC: zb_inc16(z.b, z.c, false); break;
    case DEC_BC: zb_inc16(z.b, z.c, true); break;
    case LD_BC_NN: zb_set8(z.b, (imm >> 8) & 0xFFu); zb_set8(z.c, imm & 0xFFu); break;
    default: zb_acc_step(z, op); break;
  }
}

// The register state: A, F and B..L, for pairs whose programs name neither
// SP nor the memory byte (no renaming: all six registers are held).
struct ZB6 {
  uint32_t a[8], f[8], b[8], c[8], d[8], e[8], h[8], l[8];
};
// The step on ZB6: the cases of zb_step for every instruction that names
// neither SP nor the memory byte; any other opcode leaves the state
// unchanged and must not occur.
Z80_HD void zb6_step(ZB6& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZB_REG_CASES
    default: zb_acc_step(z, op); break;
  }
}

// The wide compact state: A, F, the register pairs BC and HL and the memory
// byte.  A wide program (a pair's instructions renamed by wide_map) names no
// register but B, C, H and L and never SP; it may use the memory byte.
struct ZBW {
  uint32_t a[8], f[8], b[8], c[8], h[8], l[8], m[8];
};
#define ZBW_R(M, base) M((base) + 0, a) M((base) + 1, b) M((base) + 2, c) M((base) + 5, h) M((base) + 6, l)
#define ZBW_S(M, base) M((base) + 0, b) M((base) + 1, c) M((base) + 4, h) M((base) + 5, l) M((base) + 6, a)

// The step on ZBW: the cases of zb_step for every instruction that names no
// register but A, F, B, C, H, L (and possibly the memory byte) and not SP;
// any other opcode leaves the state unchanged and must not occur.
Z80_HD void zbw_step(ZBW& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZBW_S(ZB_LDA, LD_A_B)
    ZBW_R(ZB_LDB, LD_B_A)
    ZBW_R(ZB_LDC, LD_C_A)
    ZBW_R(ZB_LDH, LD_H_A)
    ZBW_R(ZB_LDL, LD_L_A)
    ZBW_R(ZB_LDN, LD_A_N)
    ZBW_S(ZB_ADD, ADD_A_B)
    case ADD_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, 0u); break;
    ZBW_S(ZB_ADC, ADC_A_B)
    case ADC_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, z.f[0]); break;
    ZBW_S(ZB_SUB, SUB_B)
    case SUB_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, 0u); break;
    ZBW_S(ZB_SBC, SBC_A_B)
    case SBC_A_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, z.f[0]); break;
    ZBW_S(ZB_AND, AND_B)
    case AND_N: zb_set8(t8, imm & 0xFFu); zb_and(z, t8); break;
    ZBW_S(ZB_XOR, XOR_B)
    case XOR_N: zb_set8(t8, imm & 0xFFu); zb_xor(z, t8); break;
    ZBW_S(ZB_OR, OR_B)
    case OR_N: zb_set8(t8, imm & 0xFFu); zb_or(z, t8); break;
    ZBW_S(ZB_CP, CP_B)
    case CP_N: zb_set8(t8, imm & 0xFFu); zb_cp(z, t8); break;
    ZBW_R(ZB_INC, INC_A)
    ZBW_R(ZB_DEC, DEC_A)
    ZBW_R(ZB_RLC, RLC_A)
    ZBW_R(ZB_RRC, RRC_A)
    ZBW_R(ZB_RL, RL_A)
    ZBW_R(ZB_RR, RR_A)
    ZBW_R(ZB_SLA, SLA_A)
    ZBW_R(ZB_SRA, SRA_A)
    ZBW_R(ZB_SRL, SRL_A)
    ZBW_R(ZB_SLL, SLL_A)
    ZBW_R(ZB_BIT, BIT_0_A) ZBW_R(ZB_BIT, BIT_1_A) ZBW_R(ZB_BIT, BIT_2_A) ZBW_R(ZB_BIT, BIT_3_A)
    ZBW_R(ZB_BIT, BIT_4_A) ZBW_R(ZB_BIT, BIT_5_A) ZBW_R(ZB_BIT, BIT_6_A) ZBW_R(ZB_BIT, BIT_7_A)
    ZBW_R(ZB_RES, RES_0_A) ZBW_R(ZB_RES, RES_1_A) ZBW_R(ZB_RES, RES_2_A) ZBW_R(ZB_RES, RES_3_A)
    ZBW_R(ZB_RES, RES_4_A) ZBW_R(ZB_RES, RES_5_A) ZBW_R(ZB_RES, RES_6_A) ZBW_R(ZB_RES, RES_7_A)
    ZBW_R(ZB_SET, SET_0_A) ZBW_R(ZB_SET, SET_1_A) ZBW_R(ZB_SET, SET_2_A) ZBW_R(ZB_SET, SET_3_A)
    ZBW_R(ZB_SET, SET_4_A) ZBW_R(ZB_SET, SET_5_A) ZBW_R(ZB_SET, SET_6_A) ZBW_R(ZB_SET, SET_7_A)
    case INC_BC: zb_inc16(z.b, z.c, false); break;
    case INC_HL: zb_inc16(z.h, z.l, false); break;
    case DEC_BC: zb_inc16(z.b, z.c, true); break;
    case DEC_HL: zb_inc16(z.h, z.l, true); break;
    case ADD_HL_BC: zb_hl16(z, z.c, z.b, 0); break;
    case ADD_HL_HL: zb_hl16(z, z.l, z.h, 0); break;
    case LD_BC_NN: zb_set8(z.b, (imm >> 8) & 0xFFu); zb_set8(z.c, imm & 0xFFu); break;
    case LD_HL_NN: zb_set8(z.h, (imm >> 8) & 0xFFu); zb_set8(z.l, imm & 0xFFu); break;
    case ADC_HL_BC: zb_hl16(z, z.c, z.b, 1); break;
    case ADC_HL_HL: zb_hl16(z, z.l, z.h, 1); break;
    case SBC_HL_BC: zb_hl16(z, z.c, z.b, 2); break;
    case SBC_HL_HL: zb_hl16(z, z.l, z.h, 2); break;
    case LD_A_HLI: zb_copy8(z.a, z.m); break;
    case LD_B_HLI: zb_copy8(z.b, z.m); break;
    case LD_C_HLI: zb_copy8(z.c, z.m); break;
    case LD_H_HLI: zb_copy8(z.h, z.m); break;
    case LD_L_HLI: zb_copy8(z.l, z.m); break;
    case LD_HLI_A: zb_copy8(z.m, z.a); break;
    case LD_HLI_B: zb_copy8(z.m, z.b); break;
    case LD_HLI_C: zb_copy8(z.m, z.c); break;
    case LD_HLI_H: zb_copy8(z.m, z.h); break;
    case LD_HLI_L: zb_copy8(z.m, z.l); break;
    case LD_HLI_N: zb_set8(z.m, imm & 0xFFu); break;
    case LD_A_BCI: case LD_A_DEI: zb_copy8(z.a, z.m); break;
    case LD_BCI_A: case LD_DEI_A: zb_copy8(z.m, z.a); break;
    case ADD_A_HLI: zb_copy8(t8, z.m); zb_add(z, t8, 0u); break;
    case ADC_A_HLI: zb_copy8(t8, z.m); zb_add(z, t8, z.f[0]); break;
    case SUB_HLI: zb_copy8(t8, z.m); zb_sub(z, t8, 0u); break;
    case SBC_A_HLI: zb_copy8(t8, z.m); zb_sub(z, t8, z.f[0]); break;
    case AND_HLI: zb_copy8(t8, z.m); zb_and(z, t8); break;
    case XOR_HLI: zb_copy8(t8, z.m); zb_xor(z, t8); break;
    case OR_HLI: zb_copy8(t8, z.m); zb_or(z, t8); break;
    case CP_HLI: zb_copy8(t8, z.m); zb_cp(z, t8); break;
    case INC_HLI: zb_inc(z, z.m); break;
    case DEC_HLI: zb_dec(z, z.m); break;
    case RLC_HLI: zb_rot(z, z.m, 0); break;
    case RRC_HLI: zb_rot(z, z.m, 1); break;
    case RL_HLI: zb_rot(z, z.m, 2); break;
    case RR_HLI: zb_rot(z, z.m, 3); break;
    case SLA_HLI: zb_rot(z, z.m, 4); break;
    case SRA_HLI: zb_rot(z, z.m, 5); break;
    case SRL_HLI: zb_rot(z, z.m, 6); break;
    case SLL_HLI: zb_rot(z, z.m, 7); break;
    case BIT_0_HLI: zb_bit(z, z.m, 0); break;
    case BIT_1_HLI: zb_bit(z, z.m, 1); break;
    case BIT_2_HLI: zb_bit(z, z.m, 2); break;
    case BIT_3_HLI: zb_bit(z, z.m, 3); break;
    case BIT_4_HLI: zb_bit(z, z.m, 4); break;
    case BIT_5_HLI: zb_bit(z, z.m, 5); break;
    case BIT_6_HLI: zb_bit(z, z.m, 6); break;
    case BIT_7_HLI: zb_bit(z, z.m, 7); break;
    case RES_0_HLI: z.m[0] = 0u; break;
    case RES_1_HLI: z.m[1] = 0u; break;
    case RES_2_HLI: z.m[2] = 0u; break;
    case RES_3_HLI: z.m[3] = 0u; break;
    case RES_4_HLI: z.m[4] = 0u; break;
    case RES_5_HLI: z.m[5] = 0u; break;
    case RES_6_HLI: z.m[6] = 0u; break;
    case RES_7_HLI: z.m[7] = 0u; break;
    case SET_0_HLI: z.m[0] = kZBOnes; break;
    case SET_1_HLI: z.m[1] = kZBOnes; break;
    case SET_2_HLI: z.m[2] = kZBOnes; break;
    case SET_3_HLI: z.m[3] = kZBOnes; break;
    case SET_4_HLI: z.m[4] = kZBOnes; break;
    case SET_5_HLI: z.m[5] = kZBOnes; break;
    case SET_6_HLI: z.m[6] = kZBOnes; break;
    case SET_7_HLI: z.m[7] = kZBOnes; break;
    default: zb_acc_step(z, op); break;
  }
}

// Block decoding of an ExhaustiveCheck sweep (pkg/search/verifier.go:
// 428-612), set up once per pair.  Block index fields, fastest first: SP (4
// bits, reduced sweeps that read SP), the swept registers from the last to
// the first (8 bits each in a full sweep, 5 bits indexing the representative
// values in a reduced one), carry.  Packed into two words so that it costs
// the sweep kernels two registers: register r's field position (6 bits, r =
// B, C, D, E, H, L, M; five in lo, two in hi), then in hi the swept
// registers (bit r), the SP field, the reduced sweep and the carry's
// position.  Unswept registers start at 0.
struct BDec {
  uint32_t lo, hi;
};
Z80_HD BDec bdec_make(bool spw, bool reduced, int nx, int fw, const int (&slot)[7]) {
  const int base = spw ? 4 : 0;
  uint32_t sh[7] = {0, 0, 0, 0, 0, 0, 0}, on = 0;
  for (int r = 0; r < 7; r++) {
    if (slot[r] < 0) continue;
    sh[r] = uint32_t(base + (nx - 1 - slot[r]) * fw);
    on |= 1u << r;
  }
  BDec d;
  d.lo = sh[0] | sh[1] << 6 | sh[2] << 12 | sh[3] << 18 | sh[4] << 24;
  d.hi = sh[5] | sh[6] << 6 | on << 12 | (spw ? 1u : 0u) << 19 | (reduced ? 1u : 0u) << 20 |
         uint32_t(base + nx * fw) << 21;
  return d;
}
// The initial state of block ab (A = 0); rep / repsp: the 32 representative
// register values and the 16 SP values.
Z80_HD Z80S bdec_state(const BDec& d, unsigned long long ab, const uint8_t* rep, const uint16_t* repsp) {
  const bool reduced = (d.hi >> 20) & 1u;
  uint32_t v[7];
  for (int r = 0; r < 7; r++) {
    v[r] = 0u;
    if ((d.hi >> (12 + r)) & 1u) {
      const uint32_t sh = (r < 5 ? d.lo >> (6 * r) : d.hi >> (6 * (r - 5))) & 63u;
      const uint32_t x = uint32_t(ab >> sh) & (reduced ? 31u : 255u);
      v[r] = reduced ? uint32_t(rep[x]) : x;
    }
  }
  Z80S s;
  s.a = 0;
  s.f = uint32_t(ab >> (d.hi >> 21)) & 1u;
  s.b = v[0];
  s.c = v[1];
  s.d = v[2];
  s.e = v[3];
  s.h = v[4];
  s.l = v[5];
  s.m = v[6];
  s.sp = ((d.hi >> 19) & 1u) ? uint32_t(repsp[uint32_t(ab) & 15u]) : 0u;
  return s;
}

// Block decoding for compact pairs.  A compact pair reads at most two
// registers and neither SP nor the memory byte, so its sweep is a full one:
// block index = carry above nx 8-bit fields, the last swept register in the
// lowest byte.  The initial values of the renamed B and C (the registers o0
// and o1 stand for) and the carry are then shifts and masks of the block
// index, set up once per pair: slot[r] is register r's field (-1: not
// swept; a register that is named but not read starts at 0).
struct CDec {
  uint32_t shb, mb, shc, mc, shf;
};
Z80_HD CDec cdec_make(int nx, const int (&slot)[7], int o0, int o1) {
  CDec d{0u, 0u, 0u, 0u, uint32_t(8 * nx)};
  if (o0 >= 0 && slot[o0] >= 0) {
    d.shb = uint32_t(8 * (nx - 1 - slot[o0]));
    d.mb = 0xFFu;
  }
  if (o1 >= 0 && slot[o1] >= 0) {
    d.shc = uint32_t(8 * (nx - 1 - slot[o1]));
    d.mc = 0xFFu;
  }
  return d;
}
// B, C and the carry of block ab.
Z80_HD void cdec_vals(const CDec& d, unsigned long long ab, uint32_t& vb, uint32_t& vc, uint32_t& carry) {
  const uint32_t lo = uint32_t(ab);
  vb = (lo >> d.shb) & d.mb;
  vc = (lo >> d.shc) & d.mc;
  carry = (lo >> d.shf) & 1u;
}

// Block decoding for wide compact pairs.  A wide pair reads at most four
// registers and the memory byte, never SP, so its block index (below 2^26)
// is the carry above at most five fields, 8 bits each in a full sweep and
// 5 bits indexing the representative values in a reduced one.  The initial
// values of the five wide fields (B, C, H, L as renamed, then M) are shifts
// and masks of the index: lo packs the five fields' shifts (6 bits each),
// hi the fields that are swept (bits 0..4), the reduced flag (bit 5) and the
// carry's shift (bits 6..11).  o[s]: the original register (0..5) that
// field s stands for, or -1; slot[r]: register r's sweep field (-1: not
// swept; a named register that is not read starts at 0).
struct WDec {
  uint32_t lo, hi;
};
Z80_HD WDec wdec_make(int nx, bool reduced, const int (&slot)[7], const int (&o)[4]) {
  const int fw = reduced ? 5 : 8;
  uint32_t lo = 0, on = 0;
  for (int s = 0; s < 5; s++) {
    const int r = s < 4 ? o[s] : 6;
    if (r < 0 || slot[r] < 0) continue;
    lo |= uint32_t((nx - 1 - slot[r]) * fw) << (6 * s);
    on |= 1u << s;
  }
  return WDec{lo, on | (reduced ? 32u : 0u) | uint32_t(nx * fw) << 6};
}
// The five fields and the carry of block ab.
Z80_HD void wdec_vals(const WDec& d, uint32_t ab, const uint8_t* rep, uint32_t (&v)[5], uint32_t& carry) {
  const bool reduced = (d.hi >> 5) & 1u;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int s = 0; s < 5; s++) {
    const uint32_t x = (ab >> ((d.lo >> (6 * s)) & 63u)) & (reduced ? 31u : 255u);
    v[s] = ((d.hi >> s) & 1u) ? (reduced ? uint32_t(rep[x]) : x) : 0u;
  }
  carry = (ab >> ((d.hi >> 6) & 63u)) & 1u;
}

// Planes <-> scalar states (host tests; the sweep builds planes directly).
template <class ZT>
Z80_HD void zb_from(ZT& z, const Z80S (&s)[32]) {
  for (int i = 0; i < 8; i++) {
    z.a[i] = z.f[i] = z.b[i] = z.c[i] = z.d[i] = z.e[i] = z.h[i] = z.l[i] = z.m[i] = 0;
  }
  for (int i = 0; i < 16; i++) z.sp[i] = 0;
  for (int j = 0; j < 32; j++) {
    const uint32_t bit = 1u << j;
    for (int i = 0; i < 8; i++) {
      if ((s[j].a >> i) & 1u) z.a[i] |= bit;
      if ((s[j].f >> i) & 1u) z.f[i] |= bit;
      if ((s[j].b >> i) & 1u) z.b[i] |= bit;
      if ((s[j].c >> i) & 1u) z.c[i] |= bit;
      if ((s[j].d >> i) & 1u) z.d[i] |= bit;
      if ((s[j].e >> i) & 1u) z.e[i] |= bit;
      if ((s[j].h >> i) & 1u) z.h[i] |= bit;
      if ((s[j].l >> i) & 1u) z.l[i] |= bit;
      if ((s[j].m >> i) & 1u) z.m[i] |= bit;
    }
    for (int i = 0; i < 16; i++)
      if ((s[j].sp >> i) & 1u) z.sp[i] |= bit;
  }
}
template <class ZT>
Z80_HD Z80S zb_get(const ZT& z, int j) {
  Z80S s{};
  for (int i = 0; i < 8; i++) {
    s.a |= ((z.a[i] >> j) & 1u) << i;
    s.f |= ((z.f[i] >> j) & 1u) << i;
    s.b |= ((z.b[i] >> j) & 1u) << i;
    s.c |= ((z.c[i] >> j) & 1u) << i;
    s.d |= ((z.d[i] >> j) & 1u) << i;
    s.e |= ((z.e[i] >> j) & 1u) << i;
    s.h |= ((z.h[i] >> j) & 1u) << i;
    s.l |= ((z.l[i] >> j) & 1u) << i;
    s.m |= ((z.m[i] >> j) & 1u) << i;
  }
  for (int i = 0; i < 16; i++) s.sp |= ((z.sp[i] >> j) & 1u) << i;
  return s;
}

}  // namespace z80b
