/*
 * q2d_oracle.h — CPU oracle for the Q2D explicit residual/update path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a C++ restatement of the reference Fortran
 * (open-hydra/Q2D) routines listed in each function's comment in q2d_oracle.cpp. It is the
 * checker for the CUDA path and the timed CPU baseline; the product library never links,
 * loads or calls it. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * use it.
 *
 * Parity pinning: the reference cannot be built here (no Fortran compiler; the FLINT
 * thermodynamics submodule is absent). The restatement is pinned end-to-end against the
 * reference's committed outputs (tests/golden/: ShuOsher limiter baselines written by the
 * reference binary, exact Riemann solutions) — see tests/test_oracle_golden.py.
 * Thermodynamics uses the calorically perfect single-species closure that the reference's
 * constant-cp gas tables imply (h = cp T, e = cv T, a = sqrt(gamma p / rho)), or a thermally
 * perfect single-species table (q2d_oracle_set_thermo_table). The table form is unpinned:
 * FLINT, which holds the reference's table routines, is absent, and no reference case uses a
 * variable-cp table; it is checked against closed forms of its own.
 *
 * The exported API mirrors include/q2d_gpu.h one to one (q2d_oracle_* <-> q2d_gpu_*), so a
 * test drives both through the same sequence of calls.
 */
#ifndef Q2D_ORACLE_H
#define Q2D_ORACLE_H
#include "../include/q2d_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct q2d_oracle q2d_oracle;

int  q2d_oracle_create(q2d_oracle** out, const q2d_options* opt);
int  q2d_oracle_add_case(q2d_oracle* o, int* case_id);
int  q2d_oracle_add_block(q2d_oracle* o, int case_id, int ni, int nj, const double* nodes_xy,
                          const double* cross_section, int* block_id);
int  q2d_oracle_set_bcs(q2d_oracle* o, int case_id, const q2d_bc_rec* recs, int n);
int  q2d_oracle_upload_prim(q2d_oracle* o, int block_id, const double* P);
int  q2d_oracle_set_case_time(q2d_oracle* o, int case_id, double time);
int  q2d_oracle_set_case_end(q2d_oracle* o, int case_id, long long iter_end);
int  q2d_oracle_set_thermo_table(q2d_oracle* o, int ntab, const double* h_tab, const double* cp_tab);
int  q2d_oracle_commit(q2d_oracle* o);
int  q2d_oracle_step(q2d_oracle* o, int nsteps, q2d_step_info* out);
int  q2d_oracle_case_info(q2d_oracle* o, int case_id, q2d_step_info* out);
int  q2d_oracle_download_prim(q2d_oracle* o, int block_id, double* P);
void q2d_oracle_destroy(q2d_oracle* o);
int  q2d_oracle_set_threads(int n);   /* OpenMP threads used by the cell loops; returns the count */

/* Geometry produced by Setup_Metrics, for tests: dl (2 per cell incl. ghosts, layout
 * [(i+1)+(ni+4)*(j+1)]*2+d), sur (interior, i fastest), i-face and j-face (nx, ny, len). */
int  q2d_oracle_get_geometry(q2d_oracle* o, int block_id, double* dl, double* sur,
                             double* fi, double* fj);

/* Shock sensor (SD_Tramel, Lib_Shock_Detector.f90:14-38) of every interior cell of a block,
 * i fastest, from its current state with freshly filled ghosts: the 'beta' field the reference
 * writes to its diagnostic output. */
int  q2d_oracle_shock_sensor(q2d_oracle* o, int block_id, double* beta);

/* Scalar kernels for known-answer tests. */
double q2d_oracle_limiter(int limiter, double x, double y);
double q2d_oracle_sd_tramel(double p, double p1, double p2, double p3, double p4);
/* the Riemann solver with the shock sensor beta the sensor-driven solvers blend by */
/* Thermally perfect gas on a table (h, cp at T = 0 .. ntab-1 K), for known-answer tests: out[0..3]
 * the flux of solver `riemann` (HLLC, HLLE, LLF), out[4], out[5] the sound speeds of the two
 * states, out[6] the Roe-averaged sound speed, out[7] the Roe-averaged total enthalpy, out[8]
 * rho E of primL, out[9] the pressure recovered from it (cons2prim from a guess of half its T). */
int    q2d_oracle_thermo_tab(int riemann, const q2d_options* opt, int ntab, const double* h_tab,
                             const double* cp_tab, const double* primL, const double* primR,
                             double nx, double ny, double* out);
void   q2d_oracle_riemann_sd(int riemann, const q2d_options* opt, const double* primL,
                             const double* primR, double beta, double nx, double ny, double* flux4);
void   q2d_oracle_riemann(int riemann, const q2d_options* opt, const double* primL,
                          const double* primR, double nx, double ny, double* flux4);

#ifdef __cplusplus
}
#endif
#endif
