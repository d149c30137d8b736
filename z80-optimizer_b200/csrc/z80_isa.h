// z80_isa.h -- opcode enumeration and static instruction metadata.
//
// The opcode numbering is the reference's OpCode enum
// (pkg/inst/instruction.go:50-595): 455 opcodes, memory ops from 394 on.
// Instructions are passed packed as uint32 op | imm << 16, the packing of
// the reference's GPU bridge (pkg/gpu/cuda.go:310).
#pragma once
#include <cstdint>

namespace z80b {

#define Z80B_OPCODES \
  X(LD_A_B) X(LD_A_C) X(LD_A_D) X(LD_A_E) X(LD_A_H) X(LD_A_L) X(LD_A_A) \
  X(LD_B_A) X(LD_B_B) X(LD_B_C) X(LD_B_D) X(LD_B_E) X(LD_B_H) X(LD_B_L) \
  X(LD_C_A) X(LD_C_B) X(LD_C_C) X(LD_C_D) X(LD_C_E) X(LD_C_H) X(LD_C_L) \
  X(LD_D_A) X(LD_D_B) X(LD_D_C) X(LD_D_D) X(LD_D_E) X(LD_D_H) X(LD_D_L) \
  X(LD_E_A) X(LD_E_B) X(LD_E_C) X(LD_E_D) X(LD_E_E) X(LD_E_H) X(LD_E_L) \
  X(LD_H_A) X(LD_H_B) X(LD_H_C) X(LD_H_D) X(LD_H_E) X(LD_H_H) X(LD_H_L) \
  X(LD_L_A) X(LD_L_B) X(LD_L_C) X(LD_L_D) X(LD_L_E) X(LD_L_H) X(LD_L_L) \
  X(LD_A_N) X(LD_B_N) X(LD_C_N) X(LD_D_N) X(LD_E_N) X(LD_H_N) X(LD_L_N) \
  X(ADD_A_B) X(ADD_A_C) X(ADD_A_D) X(ADD_A_E) X(ADD_A_H) X(ADD_A_L) X(ADD_A_A) \
  X(ADD_A_N) X(ADC_A_B) X(ADC_A_C) X(ADC_A_D) X(ADC_A_E) X(ADC_A_H) X(ADC_A_L) \
  X(ADC_A_A) X(ADC_A_N) X(SUB_B) X(SUB_C) X(SUB_D) X(SUB_E) X(SUB_H) \
  X(SUB_L) X(SUB_A) X(SUB_N) X(SBC_A_B) X(SBC_A_C) X(SBC_A_D) X(SBC_A_E) \
  X(SBC_A_H) X(SBC_A_L) X(SBC_A_A) X(SBC_A_N) X(AND_B) X(AND_C) X(AND_D) \
  X(AND_E) X(AND_H) X(AND_L) X(AND_A) X(AND_N) X(XOR_B) X(XOR_C) \
  X(XOR_D) X(XOR_E) X(XOR_H) X(XOR_L) X(XOR_A) X(XOR_N) X(OR_B) \
  X(OR_C) X(OR_D) X(OR_E) X(OR_H) X(OR_L) X(OR_A) X(OR_N) \
  X(CP_B) X(CP_C) X(CP_D) X(CP_E) X(CP_H) X(CP_L) X(CP_A) \
  X(CP_N) X(INC_A) X(INC_B) X(INC_C) X(INC_D) X(INC_E) X(INC_H) \
  X(INC_L) X(DEC_A) X(DEC_B) X(DEC_C) X(DEC_D) X(DEC_E) X(DEC_H) \
  X(DEC_L) X(RLCA) X(RRCA) X(RLA) X(RRA) X(DAA) X(CPL) \
  X(SCF) X(CCF) X(NEG) X(NOP) X(RLC_A) X(RLC_B) X(RLC_C) \
  X(RLC_D) X(RLC_E) X(RLC_H) X(RLC_L) X(RRC_A) X(RRC_B) X(RRC_C) \
  X(RRC_D) X(RRC_E) X(RRC_H) X(RRC_L) X(RL_A) X(RL_B) X(RL_C) \
  X(RL_D) X(RL_E) X(RL_H) X(RL_L) X(RR_A) X(RR_B) X(RR_C) \
  X(RR_D) X(RR_E) X(RR_H) X(RR_L) X(SLA_A) X(SLA_B) X(SLA_C) \
  X(SLA_D) X(SLA_E) X(SLA_H) X(SLA_L) X(SRA_A) X(SRA_B) X(SRA_C) \
  X(SRA_D) X(SRA_E) X(SRA_H) X(SRA_L) X(SRL_A) X(SRL_B) X(SRL_C) \
  X(SRL_D) X(SRL_E) X(SRL_H) X(SRL_L) X(SLL_A) X(SLL_B) X(SLL_C) \
  X(SLL_D) X(SLL_E) X(SLL_H) X(SLL_L) X(BIT_0_A) X(BIT_0_B) X(BIT_0_C) \
  X(BIT_0_D) X(BIT_0_E) X(BIT_0_H) X(BIT_0_L) X(BIT_1_A) X(BIT_1_B) X(BIT_1_C) \
  X(BIT_1_D) X(BIT_1_E) X(BIT_1_H) X(BIT_1_L) X(BIT_2_A) X(BIT_2_B) X(BIT_2_C) \
  X(BIT_2_D) X(BIT_2_E) X(BIT_2_H) X(BIT_2_L) X(BIT_3_A) X(BIT_3_B) X(BIT_3_C) \
  X(BIT_3_D) X(BIT_3_E) X(BIT_3_H) X(BIT_3_L) X(BIT_4_A) X(BIT_4_B) X(BIT_4_C) \
  X(BIT_4_D) X(BIT_4_E) X(BIT_4_H) X(BIT_4_L) X(BIT_5_A) X(BIT_5_B) X(BIT_5_C) \
  X(BIT_5_D) X(BIT_5_E) X(BIT_5_H) X(BIT_5_L) X(BIT_6_A) X(BIT_6_B) X(BIT_6_C) \
  X(BIT_6_D) X(BIT_6_E) X(BIT_6_H) X(BIT_6_L) X(BIT_7_A) X(BIT_7_B) X(BIT_7_C) \
  X(BIT_7_D) X(BIT_7_E) X(BIT_7_H) X(BIT_7_L) X(RES_0_A) X(RES_0_B) X(RES_0_C) \
  X(RES_0_D) X(RES_0_E) X(RES_0_H) X(RES_0_L) X(RES_1_A) X(RES_1_B) X(RES_1_C) \
  X(RES_1_D) X(RES_1_E) X(RES_1_H) X(RES_1_L) X(RES_2_A) X(RES_2_B) X(RES_2_C) \
  X(RES_2_D) X(RES_2_E) X(RES_2_H) X(RES_2_L) X(RES_3_A) X(RES_3_B) X(RES_3_C) \
  X(RES_3_D) X(RES_3_E) X(RES_3_H) X(RES_3_L) X(RES_4_A) X(RES_4_B) X(RES_4_C) \
  X(RES_4_D) X(RES_4_E) X(RES_4_H) X(RES_4_L) X(RES_5_A) X(RES_5_B) X(RES_5_C) \
  X(RES_5_D) X(RES_5_E) X(RES_5_H) X(RES_5_L) X(RES_6_A) X(RES_6_B) X(RES_6_C) \
  X(RES_6_D) X(RES_6_E) X(RES_6_H) X(RES_6_L) X(RES_7_A) X(RES_7_B) X(RES_7_C) \
  X(RES_7_D) X(RES_7_E) X(RES_7_H) X(RES_7_L) X(SET_0_A) X(SET_0_B) X(SET_0_C) \
  X(SET_0_D) X(SET_0_E) X(SET_0_H) X(SET_0_L) X(SET_1_A) X(SET_1_B) X(SET_1_C) \
  X(SET_1_D) X(SET_1_E) X(SET_1_H) X(SET_1_L) X(SET_2_A) X(SET_2_B) X(SET_2_C) \
  X(SET_2_D) X(SET_2_E) X(SET_2_H) X(SET_2_L) X(SET_3_A) X(SET_3_B) X(SET_3_C) \
  X(SET_3_D) X(SET_3_E) X(SET_3_H) X(SET_3_L) X(SET_4_A) X(SET_4_B) X(SET_4_C) \
  X(SET_4_D) X(SET_4_E) X(SET_4_H) X(SET_4_L) X(SET_5_A) X(SET_5_B) X(SET_5_C) \
  X(SET_5_D) X(SET_5_E) X(SET_5_H) X(SET_5_L) X(SET_6_A) X(SET_6_B) X(SET_6_C) \
  X(SET_6_D) X(SET_6_E) X(SET_6_H) X(SET_6_L) X(SET_7_A) X(SET_7_B) X(SET_7_C) \
  X(SET_7_D) X(SET_7_E) X(SET_7_H) X(SET_7_L) X(INC_BC) X(INC_DE) X(INC_HL) \
  X(INC_SP) X(DEC_BC) X(DEC_DE) X(DEC_HL) X(DEC_SP) X(ADD_HL_BC) X(ADD_HL_DE) \
  X(ADD_HL_HL) X(ADD_HL_SP) X(EX_DE_HL) X(LD_SP_HL) X(LD_BC_NN) X(LD_DE_NN) X(LD_HL_NN) \
  X(LD_SP_NN) X(ADC_HL_BC) X(ADC_HL_DE) X(ADC_HL_HL) X(ADC_HL_SP) X(SBC_HL_BC) X(SBC_HL_DE) \
  X(SBC_HL_HL) X(SBC_HL_SP) X(LD_A_HLI) X(LD_B_HLI) X(LD_C_HLI) X(LD_D_HLI) X(LD_E_HLI) \
  X(LD_H_HLI) X(LD_L_HLI) X(LD_HLI_A) X(LD_HLI_B) X(LD_HLI_C) X(LD_HLI_D) X(LD_HLI_E) \
  X(LD_HLI_H) X(LD_HLI_L) X(LD_HLI_N) X(LD_A_BCI) X(LD_A_DEI) X(LD_BCI_A) X(LD_DEI_A) \
  X(ADD_A_HLI) X(ADC_A_HLI) X(SUB_HLI) X(SBC_A_HLI) X(AND_HLI) X(XOR_HLI) X(OR_HLI) \
  X(CP_HLI) X(INC_HLI) X(DEC_HLI) X(RLC_HLI) X(RRC_HLI) X(RL_HLI) X(RR_HLI) \
  X(SLA_HLI) X(SRA_HLI) X(SRL_HLI) X(SLL_HLI) X(BIT_0_HLI) X(BIT_1_HLI) X(BIT_2_HLI) \
  X(BIT_3_HLI) X(BIT_4_HLI) X(BIT_5_HLI) X(BIT_6_HLI) X(BIT_7_HLI) X(RES_0_HLI) X(RES_1_HLI) \
  X(RES_2_HLI) X(RES_3_HLI) X(RES_4_HLI) X(RES_5_HLI) X(RES_6_HLI) X(RES_7_HLI) X(SET_0_HLI) \
  X(SET_1_HLI) X(SET_2_HLI) X(SET_3_HLI) X(SET_4_HLI) X(SET_5_HLI) X(SET_6_HLI) X(SET_7_HLI) \

enum Op : uint16_t {
#define X(n) n,
  Z80B_OPCODES
#undef X
  kNumOps
};
static_assert(kNumOps == 455, "opcode count");
static_assert(LD_A_HLI == 394, "memory ops start");

// Register bits of the read/write masks (pkg/search/verifier.go:177-188).
enum : uint16_t {
  kRegA = 1 << 0, kRegF = 1 << 1, kRegB = 1 << 2, kRegC = 1 << 3, kRegD = 1 << 4,
  kRegE = 1 << 5, kRegH = 1 << 6, kRegL = 1 << 7, kRegSP = 1 << 8, kRegM = 1 << 9
};

// Per-opcode static data, filled on the host (z80_tables.cpp) and copied to
// __constant__ memory for the kernels.
struct OpInfo {
  uint8_t size;     // encoded bytes incl. immediate (catalog.go:62-70)
  uint8_t tstates;  // catalog T-states
  uint8_t imm;      // 0 none, 1 imm8, 2 imm16
  uint8_t nopish;   // 1 for NOP and LD r,r (pruner.go:10-17)
  uint16_t reads;   // verifier.go:199-408 (opReads, with the reference's omissions)
  uint16_t writes;  // pruner.go:66-236 (opWrites; memory ops report 0)
};

inline constexpr uint16_t insn_op(uint32_t w) { return uint16_t(w & 0xFFFFu); }
inline constexpr uint16_t insn_imm(uint32_t w) { return uint16_t(w >> 16); }
inline constexpr uint32_t insn(uint16_t op, uint16_t imm = 0) { return uint32_t(op) | (uint32_t(imm) << 16); }

}  // namespace z80b
