// z80_oracle.h -- CPU restatement of the reference's candidate-verification path.
//
// TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA product
// path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// may load it.  Nothing in the product library links or calls it.
//
// It restates, in C++, the behaviour of the reference (oisee/z80-optimizer):
//   pkg/inst/instruction.go, pkg/inst/catalog.go      (ISA enum + catalog)
//   pkg/cpu/state.go, pkg/cpu/flags.go, pkg/cpu/exec.go (emulator)
//   pkg/search/{verifier,pruner,enumerator,worker,search,fingerprint}.go
//   pkg/gpu/search.go                                  (SearchGPU semantics)
//   pkg/result/{table,output}.go                       (rules + JSON)
//   cmd/z80opt/main.go:304-397,478-504                 (dead-flag + asm parsing)
//   cmd/mulopt/main.go:63-229                          (constant-multiply model)
// Parity pin: the known-answer tests of pkg/cpu/exec_test.go,
// pkg/inst/catalog_test.go, pkg/search/search_test.go and
// pkg/search/verifier_test.go, restated under tests/ and tests/golden/.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

// Opcode enumeration in the reference order (pkg/inst/instruction.go:50-595).
#define ORC_OPCODES \
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
  ORC_OPCODES
#undef X
  OpCodeCount
};

struct Instruction {
  uint16_t op;
  uint16_t imm;
};

// pkg/cpu/state.go:11-15 -- 11 bytes of architectural state.
struct State {
  uint8_t A, F, B, C, D, E, H, L;
  uint16_t SP;
  uint8_t M;
};
inline bool operator==(const State& a, const State& b) {
  return a.A == b.A && a.F == b.F && a.B == b.B && a.C == b.C && a.D == b.D &&
         a.E == b.E && a.H == b.H && a.L == b.L && a.SP == b.SP && a.M == b.M;
}
inline bool operator!=(const State& a, const State& b) { return !(a == b); }

// pkg/cpu/flags.go:4-14
constexpr uint8_t FlagC = 0x01, FlagN = 0x02, FlagP = 0x04, FlagV = 0x04,
                  Flag3 = 0x08, FlagH = 0x10, Flag5 = 0x20, FlagZ = 0x40,
                  FlagS = 0x80;

extern uint8_t Sz53Table[256], Sz53pTable[256], ParityTable[256];
extern const uint8_t HalfcarryAddTable[8], HalfcarrySubTable[8],
    OverflowAddTable[8], OverflowSubTable[8];

// pkg/inst/catalog.go:4-8
struct Info {
  std::string mnemonic;
  uint8_t bytes[2];
  int nbytes;
  int tstates;
};
extern Info Catalog[OpCodeCount];
const char* OpName(uint16_t op);

void Init();  // builds LUTs + catalog (idempotent)

bool HasImmediate(uint16_t op);
bool HasImm16(uint16_t op);
bool UsesMemory(uint16_t op);
int TStates(uint16_t op);
int ByteSize(uint16_t op);
std::string Disassemble(Instruction in);
std::string DisasmSeq(const std::vector<Instruction>& seq);  // " : " joined
int SeqByteSize(const Instruction* seq, int n);
int SeqTStates(const Instruction* seq, int n);
std::vector<uint16_t> NonImmediateOps();
std::vector<uint16_t> ImmediateOps();
std::vector<uint16_t> Imm16Ops();

// pkg/cpu/exec.go:8
int Exec(State& s, uint16_t op, uint16_t imm);

// pkg/search/verifier.go
typedef uint8_t FlagMask;
constexpr FlagMask DeadNone = 0x00, DeadUndoc = 0x28, DeadAll = 0xFF;
extern const State TestVectors[8];
extern const State MidCheckVectors[32];
State ExecSeq(State s, const Instruction* seq, int n);
bool QuickCheck(const Instruction* t, int tn, const Instruction* c, int cn);
bool MidCheck(const Instruction* t, int tn, const Instruction* c, int cn);
bool MidCheckMasked(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead);
bool QuickCheckMasked(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead);
bool ExhaustiveCheck(const Instruction* t, int tn, const Instruction* c, int cn);
bool ExhaustiveCheckMasked(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead);
FlagMask FlagDiff(const Instruction* t, int tn, const Instruction* c, int cn);
void Fingerprint(const Instruction* seq, int n, uint8_t out[80]);
bool StatesEqualMasked(const State& a, const State& b, FlagMask dead);
// Dead-register extension: registers of deadRegs (bit0..5 = B,C,D,E,H,L) are
// not compared either.
bool StatesEqualMaskedRegs(const State& a, const State& b, FlagMask dead, uint8_t deadRegs);
bool QuickCheckMaskedRegs(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead,
                          uint8_t deadRegs);
bool ExhaustiveCheckMaskedRegs(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead,
                               uint8_t deadRegs);

// Register masks (verifier.go:175-188)
enum : uint16_t {
  regA = 1 << 0, regF = 1 << 1, regB = 1 << 2, regC = 1 << 3, regD = 1 << 4,
  regE = 1 << 5, regH = 1 << 6, regL = 1 << 7, regSP = 1 << 8, regM = 1 << 9
};
uint16_t OpReads(uint16_t op);
uint16_t OpWrites(uint16_t op);
uint16_t RegsRead(const Instruction* seq, int n);
// Sweep size of ExhaustiveCheck for a pair (number of compared states).
uint64_t ExhaustiveStates(const Instruction* t, int tn, const Instruction* c, int cn);
// A CPU-time budget (seconds of the calling thread, from now; <= 0: none)
// for the thread's ExhaustiveCheck sweeps.  Once spent, sweeps report
// "not equivalent" at once and SweepBudgetSpent() is true: the results the
// thread computes from then on are void.  Bounds a timed CPU sample; the
// parity tests never set it.
void SetSweepBudget(double seconds);
bool SweepBudgetSpent();

// pkg/search/pruner.go
bool ShouldPrune(const Instruction* seq, int n);

// pkg/search/enumerator.go: the 8-bit instruction list in enumeration order
// (non-immediate ops ascending, then imm8 ops x imm 0..255).
const std::vector<Instruction>& Instructions8();
int InstructionCount8();
int InstructionCount();

// pkg/result/table.go:11-17
struct Rule {
  std::vector<Instruction> Source, Replacement;
  int BytesSaved = 0, CyclesSaved = 0;
  uint8_t DeadFlags = 0;
  uint8_t DeadRegs = 0;  // extension: registers (bit0..5 = B,C,D,E,H,L) that differ
};

struct SearchStats {
  uint64_t checked = 0;  // worker.go:134 (every enumerated candidate)
  uint64_t found = 0;
};

// worker.go:124-265 processTask (+ processTaskMasked) for ONE target.
// Appends 0..2 rules (full first, then masked) in reference order.
void ProcessTask(const Instruction* target, int tn, int maxCandLen,
                 FlagMask deadFlags, std::vector<Rule>& out, SearchStats* st);
// The same with the dead-register extension: the masked pass runs when dead
// flags or dead registers are set, compares without both, and a rule records
// the flags (OR of F differences) and registers that differ on the 8 vectors.
void ProcessTaskExt(const Instruction* target, int tn, int maxCandLen, FlagMask deadFlags, uint8_t deadRegs,
                    std::vector<Rule>& out, SearchStats* st);

// Many targets with a thread pool (worker.go:48-121).  Rules are returned
// grouped by target index order (deterministic, unlike the reference table).
std::vector<Rule> RunTasks(const std::vector<std::vector<Instruction>>& targets,
                           int maxCandLen, FlagMask deadFlags, int numWorkers,
                           SearchStats* st);

// pkg/gpu/search.go:80-199 semantics for one target against a candidate list
// (length-1 candidates): fingerprint match (80 B, dead mask on F) -> byte
// filter -> prune -> MidCheck[Masked] -> Exhaustive[Masked], all hits kept.
void SearchGPUTarget(const Instruction* target, int tn,
                     const std::vector<Instruction>& candidates,
                     FlagMask deadFlags, std::vector<Rule>& out);

// pkg/result/output.go
std::string DeadFlagDesc(uint8_t mask);
std::string WriteJSON(const std::vector<Rule>& rules);

// cmd/z80opt/main.go:304-397,478-504
bool ParseDeadFlags(const std::string& s, FlagMask* out);
bool ParseAssembly(const std::string& text, std::vector<Instruction>* out);

}  // namespace orc
