/*
 * wl_oracle.h — TEST INFRASTRUCTURE ONLY: the CPU oracle for the REWL walker hot path.
 *
 * A plain-C restatement of the reference sampler's algorithm (Faikert/
 * replica_exchange_wang_landau, C++20), written to be read beside it: each function cites
 * the reference file:line it restates.  It is pinned against the compiled reference
 * (oracle/_ref/libwlref.so, built by oracle/Makefile from the reference's own sources)
 * and against the golden fixtures in tests/golden/.  Only tests/, __graft_entry__.smoke()
 * and the CPU legs of bench.py use it; the engine never links or calls it.
 */
#ifndef WL_ORACLE_H
#define WL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/wlg.h"

typedef struct orc_couplings orc_couplings;
typedef struct orc_walker orc_walker;
typedef struct orc_result orc_result;

/* physics (src/physics.cpp) */
double orc_dipolar_pair(const double* d, const double* ai, const double* aj, double scale);
void orc_minimum_image(const double* d, const double* box, int periodic, double* out);
orc_couplings* orc_couplings_create(const wlg_system* s, char* err, size_t errlen);
void orc_couplings_destroy(orc_couplings* c);
uint64_t orc_couplings_size(const orc_couplings* c);
uint64_t orc_couplings_nnz(const orc_couplings* c);
/* Not in the reference: the update arithmetic of the engine's FP32 runs.  With on != 0,
 * add_flip_delta adds m * (double)(float)J instead of m * J; local fields and energies stay
 * FP64.  Set it after a walker's construction to follow an FP32 engine walker, whose
 * initialisation uses the FP64 couplings. */
void orc_couplings_set_update_fp32(orc_couplings* c, int on);
/* Not in the reference: the update arithmetic of the engine's BF16 runs (dense couplings): per
 * row k the scale s_k = (float) max_j |J_kj| and the values bf16(J_kj / s_k), rounded to nearest
 * even directly from the double; an accepted flip of site k adds (-2 s) * s_k * bf16(J_kj / s_k). */
void orc_couplings_set_update_bf16(orc_couplings* c, int on);
/* bfloat16 rounding (8 significant bits, exponent range of float) of a double, to nearest even,
 * in one step from the double; returned as the double it equals. */
double orc_bf16_round(double x);
/* The CSR arrays of a cutoff system: offsets[n+1], columns[nnz], values[nnz]. */
void orc_couplings_csr(const orc_couplings* c, uint64_t* offsets, uint64_t* columns, double* values);
void orc_couplings_dense(const orc_couplings* c, double* out);
void orc_local_fields(const orc_couplings* c, const int8_t* spins, double* fields);
double orc_total_energy(const orc_couplings* c, const int8_t* spins);

/* grid and windows (src/wang_landau.cpp:13-61) */
int orc_grid_bins(double emin, double emax, double width, uint64_t* bins);
int64_t orc_grid_index(double emin, double emax, double width, double energy);
int orc_partition_windows(uint64_t bins, uint64_t count, double overlap, uint64_t* out);

/* one walker (src/wang_landau.cpp:63-510) */
orc_walker* orc_walker_create(const orc_couplings* c, uint64_t id, double emin, double emax,
                              double width, uint64_t window_begin, uint64_t window_end,
                              const wlg_wl_parameters* p, uint64_t seed,
                              const int8_t* initial_spins, char* err, size_t errlen);
void orc_walker_destroy(orc_walker* w);
int orc_walker_attempt(orc_walker* w, int* accepted, char* err, size_t errlen);
int orc_walker_run(orc_walker* w, uint64_t count, char* err, size_t errlen);
void orc_walker_snapshot(const orc_walker* w, wlg_snapshot* out);
int orc_walker_restore(orc_walker* w, const wlg_snapshot* in, char* err, size_t errlen);
void orc_walker_histogram_statistics(const orc_walker* w, wlg_histogram_statistics* out);
void orc_walker_flags(const orc_walker* w, int* flat, int* covered, int* ready);
int orc_walker_begin_next_iteration(orc_walker* w, char* err, size_t errlen);
double orc_walker_exchange_log_probability(const orc_walker* a, const orc_walker* b);
int orc_walker_swap(orc_walker* a, orc_walker* b, char* err, size_t errlen);
void orc_walker_counters(const orc_walker* w, uint64_t* out);
void orc_walker_pilot(const orc_walker* w, double* squared_displacement, uint64_t* samples,
                      uint64_t* round_trips, double* representative_energies,
                      int8_t* representative_spins, uint8_t* representative_present);

/* Not in the reference: the engine's warm start (wlg_engine_warm_start and
 * wlg_engine_warm_start_continue).  Before the first attempt, the window slice of log g is
 * set from log_g (whole grid), ln f to factor (frozen at once if <= final_factor).  With
 * continue_schedule the first covered check (begin_next_iteration, src/wang_landau.cpp:
 * 389-409) halves ln f and enters the 1/t stage at once, counting round(active / factor) -
 * attempted attempts as already made: f = active / (attempted + offset) from then on
 * (update_inverse_time_factor, src/wang_landau.cpp:309-315, with the offset added). */
void orc_walker_warm_start(orc_walker* w, const double* log_g, double factor, int continue_schedule);

/* run_rewl, serial path (src/parallel.cpp:276-747) */
orc_result* orc_run_rewl(const orc_couplings* c, const wlg_run_config* config, char* err,
                         size_t errlen);
/* run_rewl with every walker warm-started (orc_walker_warm_start) after construction. */
orc_result* orc_run_rewl_warm(const orc_couplings* c, const wlg_run_config* config, const double* log_g,
                              double factor, int continue_schedule, char* err, size_t errlen);
void orc_result_destroy(orc_result* r);
void orc_result_totals(const orc_result* r, wlg_run_totals* out);
int orc_result_fragment(const orc_result* r, uint64_t w, double* log_g, uint64_t* histogram,
                        double* standard_error, uint8_t* valid);
uint64_t orc_result_walker_statistics(const orc_result* r, wlg_walker_statistics* out,
                                      uint64_t capacity);
int orc_result_sampling(const orc_result* r, uint64_t w, double* squared_displacement,
                        uint64_t* samples, uint64_t* round_trips, uint64_t* walkers);
uint64_t orc_result_representatives(const orc_result* r, double* energies, int8_t* spins,
                                    uint64_t capacity);

/* exact_enumeration (src/analysis.cpp:162-181) */
int orc_exact_enumeration(const orc_couplings* c, double emin, double emax, double width,
                          uint64_t* counts);

#endif
