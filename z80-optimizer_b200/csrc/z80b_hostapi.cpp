// z80b_hostapi.cpp -- host-side helpers exported next to the pipeline entry
// points: the pieces of pkg/inst (catalog, disassembly), pkg/result
// (JSON output) and cmd/z80opt (assembly and dead-flag parsing) a caller of
// the library needs to turn rules into the reference's output.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/z80b200.h"
#include "z80_tables.h"

using namespace z80b;

namespace {
int put_str(const std::string& s, char* buf, uint32_t cap) {
  if (buf && cap) {
    size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return int(s.size());
}
bool ok_seq(const uint32_t* s, uint32_t n) {
  for (uint32_t i = 0; i < n; i++)
    if (insn_op(s[i]) >= kNumOps) return false;
  return true;
}
void json_str(std::string& o, const std::string& s) {
  o += '"';
  for (char c : s) {
    if (c == '"') o += "\\\"";
    else if (c == '\\') o += "\\\\";
    else if (c == '<') o += "\\u003c";
    else if (c == '>') o += "\\u003e";
    else if (c == '&') o += "\\u0026";
    else o += c;
  }
  o += '"';
}
}  // namespace

extern "C" {

int z80b_op_info(uint32_t op, char* mnemonic, uint32_t cap, int* size, int* tstates, int* imm_kind,
                 int* reads, int* writes) {
  if (op >= uint32_t(kNumOps)) return Z80B_EINVAL;
  const OpInfo& o = op_table()[op];
  put_str(op_mnemonic(uint16_t(op)), mnemonic, cap);
  if (size) *size = o.size;
  if (tstates) *tstates = o.tstates;
  if (imm_kind) *imm_kind = o.imm;
  if (reads) *reads = o.reads;
  if (writes) *writes = o.writes;
  return Z80B_OK;
}

int z80b_disasm_seq(const uint32_t* seq, uint32_t n, char* buf, uint32_t cap) {
  if ((n && !seq) || !ok_seq(seq, n)) return -1;
  return put_str(disasm_seq(seq, int(n)), buf, cap);
}

int z80b_parse_assembly(const char* text, uint32_t* out, uint32_t cap) {
  if (!text) return -1;
  std::vector<uint32_t> v;
  if (!parse_assembly(text, &v)) return -1;
  for (size_t i = 0; i < v.size() && i < cap; i++) out[i] = v[i];
  return int(v.size());
}

int z80b_parse_dead_flags(const char* text, uint32_t* out) {
  uint8_t m = 0;
  if (!text || !out || !parse_dead_flags(text, &m)) return Z80B_EINVAL;
  *out = m;
  return Z80B_OK;
}

int z80b_dead_flag_desc(uint32_t mask, char* buf, uint32_t cap) {
  return put_str(dead_flag_desc(uint8_t(mask)), buf, cap);
}

int z80b_should_prune(const uint32_t* seq, uint32_t n) {
  if ((n && !seq) || !ok_seq(seq, n)) return -1;
  return should_prune(seq, int(n)) ? 1 : 0;
}

int z80b_should_prune_batch(const uint32_t* seqs, const uint8_t* lens, uint32_t stride, uint64_t n, uint8_t* out) {
  if (n && (!seqs || !lens || !out)) return Z80B_EINVAL;
  if (stride < 1 || stride > 64) return Z80B_EINVAL;
  for (uint64_t i = 0; i < n; i++) {
    const uint32_t* s = seqs + i * stride;
    const uint32_t l = lens[i];
    out[i] = (l < 1 || l > stride || !ok_seq(s, l)) ? 0xFF : (should_prune(s, int(l)) ? 1 : 0);
  }
  return Z80B_OK;
}

uint32_t z80b_pool8(uint32_t* out, uint32_t cap) {
  const auto& p = pool8();
  for (size_t i = 0; i < p.size() && i < cap; i++) out[i] = p[i];
  return uint32_t(p.size());
}

// EnumerateSequences (pkg/search/enumerator.go:280-345) over an arbitrary
// instruction pool: every length-len sequence in odometer order (position 0
// most significant), skipping those ShouldPrune rejects (search.go:344-347).
// Writes up to cap sequences (len words each) and returns the total.
uint64_t z80b_enumerate(const uint32_t* pool, uint32_t npool, uint32_t len, uint32_t* out, uint64_t cap) {
  if (!pool || !npool || len < 1 || len > 4 || !ok_seq(pool, npool)) return 0;
  uint32_t idx[4] = {0, 0, 0, 0};
  uint32_t seq[4];
  uint64_t k = 0;
  for (;;) {
    for (uint32_t i = 0; i < len; i++) seq[i] = pool[idx[i]];
    if (!should_prune(seq, int(len))) {
      if (out && k < cap) std::memcpy(out + k * len, seq, 4 * len);
      k++;
    }
    int p = int(len) - 1;
    while (p >= 0 && ++idx[p] == npool) idx[p--] = 0;
    if (p < 0) break;
  }
  return k;
}

// result.WriteJSON (pkg/result/output.go:70-90): the rules as a JSON array
// with two-space indentation.  Returns the text length (writes up to cap-1
// bytes and a terminating zero), -1 on a bad rule.
long long z80b_rules_json(const z80b_rule* rules, uint64_t n, char* buf, uint64_t cap) {
  std::string o;
  if (n == 0) {
    o = "[]\n";
  } else {
    o = "[\n";
    for (uint64_t i = 0; i < n; i++) {
      const z80b_rule& r = rules[i];
      if (r.src_len < 1 || r.src_len > 4 || r.rep_len < 1 || r.rep_len > 4) return -1;
      if (!ok_seq(r.src, uint32_t(r.src_len)) || !ok_seq(r.rep, uint32_t(r.rep_len))) return -1;
      o += "  {\n    \"source_asm\": ";
      json_str(o, disasm_seq(r.src, r.src_len));
      o += ",\n    \"replacement_asm\": ";
      json_str(o, disasm_seq(r.rep, r.rep_len));
      o += ",\n    \"source_bytes\": " + std::to_string(seq_bytes(r.src, r.src_len));
      o += ",\n    \"replacement_bytes\": " + std::to_string(seq_bytes(r.rep, r.rep_len));
      o += ",\n    \"bytes_saved\": " + std::to_string(r.bytes_saved);
      o += ",\n    \"cycles_saved\": " + std::to_string(r.cycles_saved);
      if (r.dead_flags & 0xFF) {
        char hx[8];
        std::snprintf(hx, sizeof hx, "%02X", unsigned(r.dead_flags & 0xFF));
        o += ",\n    \"dead_flags\": ";
        json_str(o, hx);
        o += ",\n    \"dead_flag_desc\": ";
        json_str(o, dead_flag_desc(uint8_t(r.dead_flags)));
      }
      o += "\n  }";
      o += (i + 1 < n) ? ",\n" : "\n";
    }
    o += "]\n";
  }
  if (buf && cap) {
    size_t k = o.size() < cap - 1 ? o.size() : cap - 1;
    std::memcpy(buf, o.data(), k);
    buf[k] = 0;
  }
  return (long long)o.size();
}

}  // extern "C"
