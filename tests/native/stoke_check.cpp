// The verifier calls of the STOKE search through the C++ host API
// (search::ExhaustiveCheck, ExhaustiveCheckMasked and FlagDiff): reads pairs
// "dead t0 t1 ... ; c0 c1 ..." (hex words, one pair per line) and prints
// "exhaustive flagdiff" per pair.  Run by tests/test_enumerate_gpu.py.
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "search_api.h"

using namespace z80opt;

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::ifstream in(argv[1]);
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string tok;
    unsigned dead = 0;
    ss >> std::hex >> dead;
    Seq t, c;
    bool cand = false;
    while (ss >> tok) {
      if (tok == ";") {
        cand = true;
        continue;
      }
      const Instruction i = Instruction::unpack(uint32_t(std::stoul(tok, nullptr, 16)));
      (cand ? c : t).push_back(i);
    }
    const bool ok = dead ? search::ExhaustiveCheckMasked(t, c, uint8_t(dead)) : search::ExhaustiveCheck(t, c);
    std::printf("%d %u\n", ok ? 1 : 0, unsigned(search::FlagDiff(t, c)));
  }
  return 0;
}
