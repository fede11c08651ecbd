// TEST INFRASTRUCTURE ONLY -- entry point of the reference-queue binaries built by
// oracle/build_ref.py.  It runs the reference's own driver (src/des.cu: des_init,
// des_run, des_finish; src/main.cc does the same) with the adapter model, then writes
// the adapter's results to the file named by argv[1]:
//   8 uint64 (num_lps, committed, windows, pending, pending_csum, error, 0, 0),
//   count uint32[num_lps], csum uint64[num_lps], ohash uint64[num_lps] (little endian).
#include <stdio.h>
#include <stdlib.h>
#include <vector>

#include "des.h"
#include "ref_adapter.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s RESULTS_FILE\n", argv[0]);
    return 2;
  }
  des_init();
  des_run();
  des_finish();
  gpq_ref_results r = {};
  std::vector<uint32_t> count(1u << 24);
  std::vector<unsigned long long> csum(1u << 24), ohash(1u << 24);
  adapter_results(&r, count.data(), csum.data(), ohash.data());
  FILE* f = fopen(argv[1], "wb");
  if (!f) return 2;
  uint64_t hdr[8] = {r.num_lps, r.committed, r.windows, r.pending, (uint64_t)r.pending_csum, r.error, 0, 0};
  fwrite(hdr, sizeof(hdr), 1, f);
  fwrite(count.data(), sizeof(uint32_t), r.num_lps, f);
  fwrite(csum.data(), sizeof(unsigned long long), r.num_lps, f);
  fwrite(ohash.data(), sizeof(unsigned long long), r.num_lps, f);
  fclose(f);
  printf("adapter: committed %llu windows %llu pending %llu error %llu\n", (unsigned long long)r.committed,
         (unsigned long long)r.windows, (unsigned long long)r.pending, (unsigned long long)r.error);
  return r.error ? 1 : 0;
}
