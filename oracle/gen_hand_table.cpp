// ORACLE — test infrastructure only.  Build step: enumerates all C(52,7)
// hands with the restated evaluator (the reference's exhaustive test,
// crates/range-solver/src/hand.rs:407-449) and writes the sorted distinct
// value table plus the per-category counts.
#include <cstdio>
#include "rs_oracle.hpp"

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s table.bin counts.txt\n", argv[0]);
    return 2;
  }
  std::vector<int32_t> table;
  uint64_t counts[9];
  oracle::hand_table_exhaustive(table, counts);
  FILE* f = fopen(argv[1], "wb");
  if (!f) return 1;
  fwrite(table.data(), 4, table.size(), f);
  fclose(f);
  f = fopen(argv[2], "w");
  if (!f) return 1;
  fprintf(f, "%zu\n", table.size());
  for (int i = 0; i < 9; ++i) fprintf(f, "%llu\n", (unsigned long long)counts[i]);
  fclose(f);
  return 0;
}
