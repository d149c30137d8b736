// Checks of the host API's rule-file functions (search_api.h): result::
// ReadJSON / FromJSON and peephole::LoadRules / Lookup / WriteTable.  Needs
// no device.  Built and run by tests/test_export.py with a scratch directory.
#include <cstdio>
#include <string>

#include "search_api.h"

using namespace z80opt;

static int fails = 0;
#define CHECK(c)                                                  \
  do {                                                            \
    if (!(c)) {                                                   \
      std::printf("FAIL line %d: %s\n", __LINE__, #c);            \
      fails++;                                                    \
    }                                                             \
  } while (0)

template <class F>
static bool throws(F f) {
  try {
    f();
  } catch (const Error& e) {
    return e.status == Z80B_EINVAL;
  }
  return false;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  // keys match case-insensitively, unknown keys and nulls are skipped
  auto v = result::ReadJSON(std::string(
      "[{\"SOURCE_ASM\": \"NEG : NEG\", \"replacement_asm\": null, \"Bytes_Saved\": 4, \"extra\": [1, {\"x\": 2}],"
      " \"cycles_saved\": 16, \"dead_flags\": \"\", \"dead_flag_desc\": \"caf\\u00e9 \\ud83d\\ude00\"}, null]"));
  CHECK(v.size() == 2);
  CHECK(v[0].SourceASM == "NEG : NEG" && v[0].ReplacementASM.empty());
  CHECK(v[0].BytesSaved == 4 && v[0].CyclesSaved == 16);
  CHECK(v[0].DeadFlagDesc == "caf\xc3\xa9 \xf0\x9f\x98\x80");
  CHECK(v[1].SourceASM.empty() && v[1].BytesSaved == 0);
  CHECK(result::ReadJSON(std::string("null")).empty());
  CHECK(result::ReadJSON(std::string(" [ ] ")).empty());
  // not an integer, trailing data, wrong types, broken text
  CHECK(throws([] { result::ReadJSON(std::string("[{\"bytes_saved\": 1.5}]")); }));
  CHECK(throws([] { result::ReadJSON(std::string("[{\"bytes_saved\": \"2\"}]")); }));
  CHECK(throws([] { result::ReadJSON(std::string("[] []")); }));
  CHECK(throws([] { result::ReadJSON(std::string("[{\"source_asm\": \"NOP\"")); }));
  CHECK(throws([] { result::ReadJSON(std::string("[{\"source_asm\": 7}]")); }));
  CHECK(throws([] { result::ReadJSON(std::string("[1]")); }));
  // back to instructions
  result::JSONRule j;
  j.SourceASM = "SUB A : LD A, 00h";
  j.ReplacementASM = "SUB A";
  j.BytesSaved = 2;
  j.CyclesSaved = 7;
  j.DeadFlags = "28";
  const result::Rule r = result::FromJSON(j);
  CHECK(r.Source.size() == 2 && r.Replacement.size() == 1 && r.DeadFlags == 0x28);
  CHECK(inst::DisasmSeq(r.Source) == "SUB A : LD A, 00h");
  j.DeadFlags = "1FF";
  CHECK(throws([&] { result::FromJSON(j); }));
  // LoadRules: the last entry of a source wins; Lookup
  const std::string path = dir + "/peep.json";
  std::FILE* f = std::fopen(path.c_str(), "w");
  std::fputs("[{\"source\": \"SLA A : RR A\", \"replacement\": \"OR A\", \"cycles_saved\": 1, \"bytes_saved\": 1},"
             " {\"source\": \"XOR A : NEG\", \"replacement\": \"XOR A\", \"cycles_saved\": 8, \"bytes_saved\": 2,"
             " \"category\": \"x\"},"
             " {\"Source\": \"SLA A : RR A\", \"replacement\": \"OR A\", \"cycles_saved\": 12, \"bytes_saved\": 3}]",
             f);
  std::fclose(f);
  const peephole::Table t = peephole::LoadRules(path);
  CHECK(t.size() == 2);
  const peephole::Rule* p = peephole::Lookup(t, "SLA A : RR A");
  CHECK(p && p->Replacement == "OR A" && p->CyclesSaved == 12 && p->BytesSaved == 3);
  CHECK(peephole::Lookup(t, "NOP : NOP") == nullptr);
  CHECK(throws([&] { peephole::LoadRules(dir + "/missing.json"); }));
  // WriteTable quotes keys and values as Go %q does
  const std::string out = dir + "/table.go";
  f = std::fopen(out.c_str(), "w");
  peephole::WriteTable(f, {{"LD A, \"x\\", peephole::Rule{"NOP", 4, 1}}}, "t.json", "T");
  std::fclose(f);
  f = std::fopen(out.c_str(), "r");
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  std::fclose(f);
  CHECK(text.find("\t\"LD A, \\\"x\\\\\": {\"NOP\", 4, 1},\n") != std::string::npos);
  CHECK(text.find("var T = map[string]Rule{\n") != std::string::npos);
  if (fails) return 1;
  std::printf("OK\n");
  return 0;
}
