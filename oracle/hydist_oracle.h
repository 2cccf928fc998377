/* hydist_oracle.h -- TEST INFRASTRUCTURE ONLY: C interface of the FP64 CPU
 * restatement of the Hydist_C time step used to check the CUDA path. */
#ifndef HYDIST_ORACLE_H
#define HYDIST_ORACLE_H

#include "../include/hydist_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleSim OracleSim;

const char* oracle_last_error(void);
OracleSim* oracle_create(const HydistScenario* sc, const HydistParams* p,
                         const HydistOptions* o, int nthreads);
void oracle_destroy(OracleSim* s);
void oracle_set_race_mode(OracleSim* s, int race_new);
int oracle_step(OracleSim* s, int nsteps);
double oracle_time(OracleSim* s);
void oracle_set_time(OracleSim* s, double t);
int oracle_rescan_segments(OracleSim* s);
int oracle_get(OracleSim* s, int field, void* out);
int oracle_set(OracleSim* s, int field, const void* in);
int oracle_get_segments(OracleSim* s, int kind, int* dau, int* cuoi, int* moc);
int oracle_get_boundary(OracleSim* s, double* ubt, double* ubp, double* vbt,
                        double* vbd, double* hi, double* hmax4);
int oracle_thomas(int n, const double* dl, const double* d, const double* du,
                  const double* b, double* x);
int oracle_thomas_batched(const double* dl, const double* d, const double* du,
                          const double* b, double* x, const int* offsets,
                          const int* lengths, int nsys, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
