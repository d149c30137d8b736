// z80_bits_core.cuh -- the full bit-sliced state (ZB) and its step
// (zb_step), with the plane word type ZW left to the includer: z80_bits.cuh
// includes it with ZW = uint32_t (32 states per word) for the kernels, and
// the dependency derivation in z80_tables.cpp with a word type that carries,
// instead of bits, the set of input fields a plane depends on.  No include
// guard: it is meant to be included once per word type, each time inside a
// namespace that defines ZW and sees z80_exec.cuh's names.

struct ZB {
  ZW a[8], f[8], b[8], c[8], d[8], e[8], h[8], l[8], m[8];
  ZW sp[16];
};
constexpr uint32_t kZBOnes = 0xFFFFFFFFu;

#if defined(__CUDA_ARCH__)  // device pass only: host compilers do not know the pragma
#define ZB_UNROLL _Pragma("unroll")
#else
#define ZB_UNROLL
#endif

Z80_HD ZW zb_maj(ZW x, ZW y, ZW z) { return (x & y) | (z & (x | y)); }
Z80_HD ZW zb_any(const ZW (&r)[8]) {
  return (r[0] | r[1] | r[2] | r[3]) | (r[4] | r[5] | r[6] | r[7]);
}
// P/V after logic ops: set when the number of one bits is even.
Z80_HD ZW zb_even(const ZW (&r)[8]) {
  return ~((r[0] ^ r[1] ^ r[2] ^ r[3]) ^ (r[4] ^ r[5] ^ r[6] ^ r[7]));
}
Z80_HD void zb_set8(ZW (&r)[8], uint32_t v) {
  ZB_UNROLL for (int i = 0; i < 8; i++) r[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
}
Z80_HD void zb_copy8(ZW (&d)[8], const ZW (&s)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) d[i] = s[i];
}
// S, Z, 5, 3 of a result (z_sz53), P/V and H, N cleared.
template <class ZT>
Z80_HD void zb_sz53p(ZT& z, const ZW (&r)[8], ZW carry) {
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
Z80_HD ZW zb_adder8(const ZW (&x)[8], const ZW (&y)[8], ZW cin, ZW (&r)[8],
                          ZW* c4) {
  ZW c = cin;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    if (i == 4) *c4 = c;
    r[i] = x[i] ^ y[i] ^ c;
    c = zb_maj(x[i], y[i], c);
  }
  return c;
}
template <class ZT>
Z80_HD void zb_add(ZT& z, const ZW (&v)[8], ZW cin) {
  ZW r[8], c4 = 0;
  const ZW co = zb_adder8(z.a, v, cin, r, &c4);
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
Z80_HD ZW zb_suber8(const ZW (&x)[8], const ZW (&v)[8], ZW bin, ZW (&r)[8],
                          ZW* h) {
  ZW nv[8];
  ZB_UNROLL for (int i = 0; i < 8; i++) nv[i] = ~v[i];
  ZW c4 = 0;
  const ZW co = zb_adder8(x, nv, ~bin, r, &c4);
  *h = ~c4;  // bit 4 of x ^ v ^ r
  return ~co;
}
template <class ZT>
Z80_HD void zb_sub(ZT& z, const ZW (&v)[8], ZW bin) {
  ZW r[8], h = 0;
  const ZW borrow = zb_suber8(z.a, v, bin, r, &h);
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
Z80_HD void zb_cp(ZT& z, const ZW (&v)[8]) {
  ZW r[8], h = 0;
  const ZW borrow = zb_suber8(z.a, v, 0u, r, &h);
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
Z80_HD void zb_and(ZT& z, const ZW (&v)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) z.a[i] &= v[i];
  zb_sz53p(z, z.a, 0u);
  z.f[4] = kZBOnes;
}
template <class ZT>
Z80_HD void zb_xor(ZT& z, const ZW (&v)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) z.a[i] ^= v[i];
  zb_sz53p(z, z.a, 0u);
}
template <class ZT>
Z80_HD void zb_or(ZT& z, const ZW (&v)[8]) {
  ZB_UNROLL for (int i = 0; i < 8; i++) z.a[i] |= v[i];
  zb_sz53p(z, z.a, 0u);
}
// z_inc / z_dec
template <class ZT>
Z80_HD void zb_inc(ZT& z, ZW (&r)[8]) {
  ZW c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const ZW t = r[i];
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
Z80_HD void zb_dec(ZT& z, ZW (&r)[8]) {
  z.f[4] = ~(r[0] | r[1] | r[2] | r[3]);
  ZW c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const ZW t = r[i];
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
  const ZW lo_gt9 = z.a[3] & (z.a[2] | z.a[1]);
  const ZW hi_gt9 = z.a[7] & (z.a[6] | z.a[5]);
  const ZW hi_eq9 = z.a[7] & ~z.a[6] & ~z.a[5] & z.a[4];
  const ZW gt99 = hi_gt9 | (hi_eq9 & lo_gt9);
  const ZW add6 = z.f[4] | lo_gt9;
  const ZW add60 = z.f[0] | gt99;
  const ZW carry = z.f[0] | gt99;
  ZW v[8] = {0u, add6, add6, 0u, 0u, add60, add60, 0u};
  ZT za = z, zs = z;
  zb_add(za, v, 0u);
  zb_sub(zs, v, 0u);
  const ZW n = z.f[1];
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    z.a[i] = (zs.a[i] & n) | (za.a[i] & ~n);
    z.f[i] = (zs.f[i] & n) | (za.f[i] & ~n);
  }
  z.f[0] = carry;
  z.f[2] = zb_even(z.a);
}
// ---- CB rotates and shifts; results into r, flags from the new value
template <class ZT>
Z80_HD void zb_rot(ZT& z, ZW (&r)[8], int kind) {
  ZW n[8], co = 0;
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
Z80_HD void zb_bit(ZT& z, const ZW (&r)[8], int bit) {
  const ZW nb = ~r[bit];
  z.f[1] = 0;
  z.f[2] = nb;
  z.f[3] = r[3];
  z.f[4] = kZBOnes;
  z.f[5] = r[5];
  z.f[6] = nb;
  z.f[7] = bit == 7 ? r[7] : 0u;
}
// ---- 16-bit arithmetic on (hi, lo) register pairs
Z80_HD void zb_inc16(ZW (&hi)[8], ZW (&lo)[8], bool dec) {
  ZW c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const ZW t = lo[i];
    lo[i] = t ^ c;
    c = (dec ? ~t : t) & c;
  }
  ZB_UNROLL for (int i = 0; i < 8; i++) {
    const ZW t = hi[i];
    hi[i] = t ^ c;
    c = (dec ? ~t : t) & c;
  }
}
Z80_HD void zb_incsp(ZW (&sp)[16], bool dec) {
  ZW c = kZBOnes;
  ZB_UNROLL for (int i = 0; i < 16; i++) {
    const ZW t = sp[i];
    sp[i] = t ^ c;
    c = (dec ? ~t : t) & c;
  }
}
// HL + v (+ carry) / HL - v - carry over 16 planes, in place; kind 0 ADD,
// 1 ADC, 2 SBC.  v is given as its low and high byte planes (vlo, vhi),
// which may be HL's own: bit i of both operands is read before bit i of HL
// is written.
template <class ZT>
Z80_HD void zb_hl16(ZT& z, const ZW* vlo, const ZW* vhi, int kind) {
  ZW c = kind == 0 ? 0u : (kind == 1 ? z.f[0] : ~z.f[0]), c12 = 0, nz = 0, x15 = 0, v15 = 0;
  ZB_UNROLL for (int i = 0; i < 16; i++) {
    ZW& xr = i < 8 ? z.l[i] : z.h[i - 8];
    const ZW vi = i < 8 ? vlo[i] : vhi[i - 8];
    const ZW x = xr, y = kind == 2 ? ~vi : vi;
    if (i == 12) c12 = c;
    if (i == 15) {
      x15 = x;
      v15 = vi;
    }
    const ZW r = x ^ y ^ c;
    c = zb_maj(x, y, c);
    xr = r;
    nz |= r;
  }
  const ZW r15 = z.h[7];
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
#define ZB_ADD(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_add(z, v_, 0u); } break;
#define ZB_ADC(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_add(z, v_, z.f[0]); } break;
#define ZB_SUB(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_sub(z, v_, 0u); } break;
#define ZB_SBC(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_sub(z, v_, z.f[0]); } break;
#define ZB_AND(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_and(z, v_); } break;
#define ZB_XOR(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_xor(z, v_); } break;
#define ZB_OR(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_or(z, v_); } break;
#define ZB_CP(o, r) case (o): { ZW v_[8]; zb_copy8(v_, z.r); zb_cp(z, v_); } break;
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
  ZW t8[8];
  switch (op) {
    case RLCA: {
      const ZW o7 = z.a[7];
      for (int i = 7; i > 0; i--) z.a[i] = z.a[i - 1];
      z.a[0] = o7;
      z.f[0] = o7; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case RRCA: {
      const ZW o0 = z.a[0];
      for (int i = 0; i < 7; i++) z.a[i] = z.a[i + 1];
      z.a[7] = o0;
      z.f[0] = o0; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case RLA: {
      const ZW o7 = z.a[7];
      for (int i = 7; i > 0; i--) z.a[i] = z.a[i - 1];
      z.a[0] = z.f[0];
      z.f[0] = o7; z.f[1] = 0; z.f[3] = z.a[3]; z.f[4] = 0; z.f[5] = z.a[5];
    } break;
    case RRA: {
      const ZW o0 = z.a[0];
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
        const ZW dd = z.d[i], ee = z.e[i]; \
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
  ZW t8[8];
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

