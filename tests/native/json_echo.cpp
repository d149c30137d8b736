// Echoes a rules JSON file through result::ReadJSON: one line per rule, the
// eight fields tab-separated with their strings hex-encoded (byte for byte),
// or "ERROR" when the reader rejects the file.  Used by tests/test_export.py
// to compare the reader with Python's json module on generated files.
#include <cstdio>

#include "search_api.h"

using namespace z80opt;

static void hex(const std::string& s) {
  for (unsigned char c : s) std::printf("%02x", c);
  std::printf("\t");
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  try {
    const auto rules = result::ReadJSON(f);
    for (const auto& r : rules) {
      hex(r.SourceASM);
      hex(r.ReplacementASM);
      std::printf("%d\t%d\t%d\t%d\t", r.SourceBytes, r.ReplacementBytes, r.BytesSaved, r.CyclesSaved);
      hex(r.DeadFlags);
      hex(r.DeadFlagDesc);
      std::printf("\n");
    }
  } catch (const Error&) {
    std::printf("ERROR\n");
  }
  std::fclose(f);
  return 0;
}
