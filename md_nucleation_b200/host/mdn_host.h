/*
 * mdn_host.h -- the C++ host of the engine: the reference program's input
 * script, molecule files, initial placement, run cadence and output files,
 * driving libmdn.so through include/mdn.h.
 *
 * A condition file in the reference's format (MD::readCondFile,
 * src/initialization/setCondition.cpp:4-254) names the ion and vapor files
 * (Variables::readIonFile / readVaporFile, src/initialization/readIonFile.cpp,
 * readVaporFile.cpp), the gas, T, p, dt, the step counts, the output cadence
 * and the Interactions keywords.  mdnh_load reads them, places the molecules
 * (MD::initialization_gas / initialization_vapor, Variables::ionInitial) and
 * builds the engine's replica descriptor; mdnh_run runs a batch of such
 * systems on one GPU with MD::run's cadence (src/run.cpp:17-74) and writes the
 * reference's files: <Output>_<n>.dump (MD::export_dump_close), K_<n>.dat and
 * U_<n>.dat (MD::display), ion_<T>_<n>.dat (MD::output), vapor_in_<n>.dat and
 * vapor_out_<n>.dat (MD::Ovin / MD::Ovout).
 */
#ifndef MDN_HOST_H
#define MDN_HOST_H

#include "mdn.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdnh_system mdnh_system;

/* The settings of a condition file that are not part of the descriptor. */
typedef struct mdnh_settings {
  long long total_steps;   /* TotalSteps                                   */
  long long relax_steps;   /* RelaxSteps                                   */
  int observe;             /* Output <prefix> <OBSERVE>                    */
  int calc_number;         /* the calculation number of the output names   */
  double pressure;         /* Pressure (Pa)                                */
  int n_gas, n_vapor;      /* Gas <kind> <n>, Vapor <file> <n>             */
  int gas_kind;            /* MDN_GAS_*                                    */
  unsigned interactions;   /* MDN_I_* bits                                 */
  int nvt_mode;            /* MDN_NVT_* of NVTion                          */
  double nvt_temperature;
  double box;              /* d_size (A)                                   */
} mdnh_settings;

/* Reads the condition file and the files it names, places the molecules and
 * builds the descriptor, on the CPU.  calc_number names the outputs (as the
 * reference's second argument) and, with seed, keys the placement and the
 * engine's random streams: seed 0 takes 0x4D444E55 + calc_number.
 * reference_masses = 1 divides gas centres of mass by the reference's
 * molecular masses (src/constants.hpp:34) instead of the atom-mass sum.     */
int mdnh_load(const char* condition_file, int calc_number, unsigned long long seed, int reference_masses,
              mdnh_system** out);
/* As mdnh_load, with the gas and vapor placed on GPU place_device by
 * mdn_place (counter-based stream, include/mdn.h) when place_device >= 0;
 * -1 places them on the CPU as mdnh_load does.  Both follow the reference's
 * acceptance rule; the two streams differ, so the systems do too. */
int mdnh_load_ex(const char* condition_file, int calc_number, unsigned long long seed, int reference_masses,
                 int place_device, mdnh_system** out);
void mdnh_free(mdnh_system* s);
const char* mdnh_last_error(void);

const mdn_replica_desc* mdnh_desc(const mdnh_system* s);
int mdnh_get_settings(const mdnh_system* s, mdnh_settings* out);
/* Atom-type name as the reference prints it in dumps ("C", "H(v)", "N(g)"...). */
const char* mdnh_type_name(const mdnh_system* s, int type);
/* Names of the output files. */
const char* mdnh_dump_path(const mdnh_system* s);

/* One frame of MD::export_dump_close (src/output/output.cpp:133-170): rows
 * of in-domain atoms (ion first, then molecules in order), positions shifted
 * by -shift (the ion centre when dump_fix is on, as in the reference).      */
int mdnh_write_dump_frame(const mdnh_system* s, const char* path, int timestep, int n_rows, const int* type,
                          const double* x, const double* v, const double* shift);

/* Runs n systems as one batch on one GPU: RelaxSteps with the NVTion
 * thermostat, the re-initialisation of src/run.cpp:40-56 (recentre, rebuild,
 * NVE), then TotalSteps, writing every system's output files at the
 * reference's cadence.  verbose = 1 prints MD::display's summary of system 0. */
int mdnh_run(mdnh_system* const* systems, int n, const mdn_options* opt, int verbose);

#ifdef __cplusplus
}
#endif
#endif /* MDN_HOST_H */
