/*
 * mdn_run -- the reference program's command line (src/main.cpp:9-33) on the
 * engine: mdn_run <condition file> <calculation number> [replicas]
 *
 * The reference runs one replica per OpenMP thread, calculation numbers n,
 * n+1, ...; here every replica goes into one batch on one GPU.  The replica
 * count is the third argument, else OMP_NUM_THREADS, else 1.  Each replica
 * writes the reference's output files under its own calculation number.
 * The molecules are placed on the GPU (mdn_place); MDN_PLACEMENT=cpu places
 * them on the CPU instead.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "mdn_host.h"

int main(int argc, char** argv) {
  if (argc < 3 || argc > 4) {
    fprintf(stderr,
            "usage: mdn_run <condition file> <calculation number> [replicas]\n"
            "  runs the replicas (calculation numbers n, n+1, ...) as one batch on one GPU\n"
            "  MDN_PLACEMENT=cpu places the molecules on the CPU (default: on the GPU)\n");
    return 2;
  }
  const int calc = atoi(argv[2]);
  int replicas = 1;
  if (argc == 4) replicas = atoi(argv[3]);
  else if (getenv("OMP_NUM_THREADS")) replicas = atoi(getenv("OMP_NUM_THREADS"));
  if (replicas < 1) {
    fprintf(stderr, "mdn_run: replica count must be >= 1\n");
    return 2;
  }
  mdn_options opt;
  mdn_default_options(&opt);
  const char* pl = getenv("MDN_PLACEMENT");
  const int place_device = (pl && strcmp(pl, "cpu") == 0) ? -1 : opt.device;
  std::vector<mdnh_system*> sys(replicas, nullptr);
  int rc = 0;
  for (int r = 0; r < replicas && !rc; r++) {
    rc = mdnh_load_ex(argv[1], calc + r, 0, 0, place_device, &sys[r]);
    if (rc) fprintf(stderr, "mdn_run: %s\n", mdnh_last_error());
  }
  if (!rc) {
    mdnh_settings st;
    mdnh_get_settings(sys[0], &st);
    printf("mdn_run: %d replica(s), %d gas + %d vapor molecules each, box %.1f A, %lld relax + %lld steps\n",
           replicas, st.n_gas, st.n_vapor, st.box, st.relax_steps, st.total_steps);
    rc = mdnh_run(sys.data(), replicas, &opt, 1);
    if (rc) fprintf(stderr, "mdn_run: %s\n", mdnh_last_error());
  }
  for (mdnh_system* s : sys) mdnh_free(s);
  return rc ? 1 : 0;
}
