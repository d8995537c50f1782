// hst_oracle: runs a deck through the oracle's restatement of program hst
// (src/hst.f90) and writes the final field as a CPL file.  Test
// infrastructure only.
//   hst_oracle <deck> [out.fld] [max_steps]
#include <cstdio>
#include <cstdlib>
#include "hst_oracle.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: hst_oracle deck [out.fld] [max_steps]\n");
    return 2;
  }
  ora_params p;
  if (ora_read_deck(argv[1], &p) != 0) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 1;
  }
  const char* out = argc > 2 ? argv[2] : "Dati.cart.out";
  long maxs = argc > 3 ? std::atol(argv[3]) : 1L << 60;
  ora_sim* s = ora_create(&p);
  ora_start(s);
  long n = ora_run(s, maxs);
  std::printf("oracle: %ld steps, time %.17g\n", n, ora_get_time(s));
  int rc = ora_restart_write(s, out);
  ora_destroy(s);
  return rc;
}
