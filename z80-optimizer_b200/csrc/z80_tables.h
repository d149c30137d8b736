// z80_tables.h -- host-side instruction catalog and static analysis.
//
// The catalog (mnemonics, encodings, T-states) is the reference's
// pkg/inst/catalog.go data; the read/write masks are the reference's
// opReads/opWrites (pkg/search/verifier.go:199-408, pruner.go:66-236),
// including their omissions, because pruning and sweep selection depend on
// them bit for bit.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "z80_isa.h"

namespace z80b {

const OpInfo* op_table();                 // kNumOps entries

// How an instruction's outputs depend on the input value of A (derived by
// running the step function on every A value of sampled input states):
//   kADepends    some output other than A, or A itself, depends on A
//   kAPass       A passes through unchanged, nothing else depends on A
//   kAOverwrite  A is written from other inputs, nothing depends on A
enum AClass : uint8_t { kADepends = 0, kAPass = 1, kAOverwrite = 2 };
const uint8_t* op_aclass();               // kNumOps entries
// Folds the classes over a sequence: 0 when some output depends on the input
// A; else 1 (A is overwritten) or 3 (A passes through to the output).
uint32_t seq_aflow(const uint32_t* s, int n);
// Which input fields each output field of an instruction depends on.  A
// field is a bit of a mask laid out like the register read masks: A bit 0,
// B..L bits 2..7, SP bit 8, the memory byte bit 9, and the flag bits F0..F7
// one by one at bits 16..23 (kDepF0 + k).  deps[op][g] is the mask of input
// fields that output field g can depend on, g a bit position of that layout
// (entries of unused positions are 0); an output the instruction leaves
// alone depends on itself.  Derived by running the bit-sliced step
// (z80_bits_core.cuh) on planes that carry, instead of bits, the set of
// input fields they were computed from: a sound over-approximation (every
// real dependency is in the set).
constexpr int kDepF0 = 16, kDepFields = 24;
const uint32_t (*op_deps())[kDepFields];  // kNumOps rows
// Input fields that the outputs in `out` (a mask of the layout above) of
// the sequence s can depend on.
uint32_t seq_relevant(const uint32_t* s, int n, uint32_t out);
// Instructions that leave A exactly as it was (from the same run: every A
// plane is still the input plane, moved by nothing but copies); kNumOps
// entries, 1 = keeps A.
const uint8_t* op_keeps_a();
bool seq_keeps_a(const uint32_t* s, int n);
// Two values of A decide the pair's ExhaustiveCheck when no compared output
// but A depends on the input A (cmp: the compared outputs, layout above) and
// each program either keeps A or computes its A from other inputs: every
// other output is then the same for all values of A, and A_out is A_in or a
// constant in each program (the argument of the A-independent sweeps, now
// under the dead flags and registers).
bool pair_a_free(const uint32_t* t, int tn, const uint32_t* c, int cn, uint32_t cmp);
// The same for every register and the memory byte (read-mask bits): kNumOps
// entries of the fields the instruction leaves exactly as they were, and
// their AND over a sequence.
const uint16_t* op_keeps();
uint32_t seq_keeps(const uint32_t* s, int n);
// Swept registers (`swept`, B..L and M bits) that both programs keep
// exactly and that no other compared output depends on: their compared
// outputs are equal whatever their value, so one value decides.
uint32_t pair_kept_out(const uint32_t* t, int tn, const uint32_t* c, int cn, uint32_t cmp, uint32_t swept);
const char* op_mnemonic(uint16_t op);     // "ADD A, n" style with placeholders
// The instruction that does op's work with the 8-bit registers renamed:
// register r (0..5 = B, C, D, E, H, L) plays the part of map[r] (map is a
// permutation).  A, F, SP and the memory byte keep their parts; a register
// pair that op uses as one (BC, DE, HL outside parentheses) must map onto a
// pair in order.  Returns -1 when the catalog has no such instruction (HL as
// the fixed operand of ADD/ADC/SBC HL, EX DE,HL or LD SP,HL renamed away, or
// a pair split).  Memory operands ((HL), (BC), (DE)) stay as they are: the
// step function's memory byte does not depend on the address registers.
int op_rename(uint16_t op, const uint8_t (&map)[6]);
// Registers an instruction names, read or written: bit r (r = 0..5) for B,
// C, D, E, H, L (a register pair counts both halves), bit 6 for the memory
// byte (a parenthesised operand), bit 7 for SP.  A and F are left out.  The
// catalog's instructions use no other registers implicitly.
uint8_t op_regs(uint16_t op);
// A pair whose two programs name at most two of B..L and neither SP nor the
// memory byte, with its registers renamed onto B and C (pairs used as pairs
// onto BC): map[r] is register r's new place, tw/cw the renamed programs.
// False when the pair names more, or a renaming does not exist.
bool compact_map(const uint32_t* t, int tn, const uint32_t* c, int cn, uint8_t (&map)[6], uint32_t* tw,
                 uint32_t* cw);
// The renaming compact_map uses for a set of at most two of B..L (bit r =
// register r): the set's registers onto B and C (in order), the others onto
// the places left.
void compact_set_map(uint8_t set, uint8_t (&map)[6]);
// The same mapping as tables for the device, one entry per set of at most
// two registers (22 sets): id_of_set[set] = 1 + entry (0 for larger sets),
// ren[entry][op] the renamed opcode or -1, orig[entry][s] the original
// register (0..5) that plays B (s = 0) or C (s = 1), or -1, and op_regs of
// every opcode.
constexpr int kCompactSets = 22;
struct CompactTables {
  int16_t ren[kCompactSets][kNumOps];
  int8_t orig[kCompactSets][2];
  uint8_t id_of_set[64];
  uint8_t opregs[kNumOps];
};
const CompactTables& compact_tables();
// The wide compact state holds A, F, B, C, H, L and the memory byte.  A pair
// whose programs name at most four of B..L and not SP is renamed onto B, C,
// H and L: a register pair used as one (both halves in the set) onto BC or
// HL, keeping its own place when that is BC or HL; single registers keep
// their place when it is B, C, H or L and free, else take the first free of
// them.  False when the pair names more, or a renamed opcode does not exist.
bool wide_map(const uint32_t* t, int tn, const uint32_t* c, int cn, uint8_t (&map)[6], uint32_t* tw, uint32_t* cw);
void wide_set_map(uint8_t set, uint8_t (&map)[6]);
// The wide renaming as tables for the device, one entry per set of at most
// four registers (57 sets): id_of_set[set] = 1 + entry (0 for larger sets),
// ren[entry][op] the renamed opcode or -1, orig[entry][s] the original
// register (0..5) that plays B, C, H, L (s = 0..3), or -1.
constexpr int kWideSets = 57;
struct WideTables {
  int16_t ren[kWideSets][kNumOps];
  int8_t orig[kWideSets][4];
  uint8_t id_of_set[64];
};
const WideTables& wide_tables();
const uint8_t* op_encoding(uint16_t op, int* n);
std::string disassemble(uint32_t insn);   // catalog.go:73-127
std::string disasm_seq(const uint32_t* seq, int n);  // " : " joined

inline int seq_bytes(const uint32_t* s, int n) {
  int b = 0;
  for (int i = 0; i < n; i++) b += op_table()[insn_op(s[i])].size;
  return b;
}
inline int seq_tstates(const uint32_t* s, int n) {
  int t = 0;
  for (int i = 0; i < n; i++) t += op_table()[insn_op(s[i])].tstates;
  return t;
}

// pkg/search/pruner.go:7-35
bool should_prune(const uint32_t* seq, int n);

// The 8-bit instruction list in the enumeration order of
// pkg/search/enumerator.go:319-345: non-immediate opcodes ascending, then
// the imm8 opcodes ascending with imm 0..255.  4531 entries.
const std::vector<uint32_t>& pool8();
// EnumerateFirstOp order (enumerator.go:358-374): pool8 then the imm16 ops
// with imm 0..65535.  266,675 entries.
std::vector<uint32_t> first_op_pool();

// Sweep shape of ExhaustiveCheck for a pair (verifier.go:159-171,428-476):
// kind 0 = A x carry (512 states), 1 = full sweep of n extra 8-bit
// registers (512 * 256^n states), 2 = reduced sweep (512 * 32^n [* 16]).
struct Sweep {
  int kind;
  int nextra;         // extra 8-bit registers swept
  uint8_t regs[7];    // 0..6 = B,C,D,E,H,L,M in that order
  bool sp;            // reduced sweep includes 16 SP values
  uint64_t states;
};
Sweep sweep_for(uint16_t reads);
uint16_t seq_reads(const uint32_t* s, int n);

// Fixed test vectors, packed as {A|F<<8|B<<16|C<<24, D|E<<8|H<<16|L<<24,
// SP|M<<16}: the 8 QuickCheck vectors (pkg/search/verifier.go:19-28) and the
// 32 MidCheck vectors (verifier.go:35-72).  Reduced-sweep representative
// values (verifier.go:537-542) and SP values (verifier.go:564-567).
const uint32_t (*qc_vectors())[3];
const uint32_t (*mid_vectors())[3];
const uint8_t* rep_values();    // 32
const uint16_t* rep_sp();       // 16

// cmd/z80opt/main.go:305-322 and 325-397,478-504
bool parse_dead_flags(const std::string& s, uint8_t* out);
bool parse_assembly(const std::string& text, std::vector<uint32_t>* out);
// pkg/result/output.go:93-129
std::string dead_flag_desc(uint8_t mask);

}  // namespace z80b
