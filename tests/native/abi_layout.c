/* Prints sizeof/offsetof of every struct in include/wlg.h as JSON (test_abi.py compares
 * them with the ctypes mirror in replica_exchange_wang_landau_b200/_abi.py). */
#include <stddef.h>
#include <stdio.h>

#include "../../include/wlg.h"

#define F(T, m) printf("\"%s.%s\": %zu, ", #T, #m, offsetof(T, m))
#define S(T) printf("\"%s\": %zu, ", #T, sizeof(T))

int main(void) {
    printf("{");
    S(wlg_system); F(wlg_system, n); F(wlg_system, positions); F(wlg_system, axes); F(wlg_system, box);
    F(wlg_system, periodic); F(wlg_system, coupling_scale); F(wlg_system, cutoff);
    S(wlg_couplings); F(wlg_couplings, n); F(wlg_couplings, dense); F(wlg_couplings, nnz);
    F(wlg_couplings, row_offsets); F(wlg_couplings, columns); F(wlg_couplings, values);
    S(wlg_wl_parameters); F(wlg_wl_parameters, flatness); F(wlg_wl_parameters, minimum_visits);
    F(wlg_wl_parameters, final_factor); F(wlg_wl_parameters, check_interval_attempts);
    F(wlg_wl_parameters, force_accept_after_attempts); F(wlg_wl_parameters, inverse_time_enabled);
    F(wlg_wl_parameters, initialization_max_attempts); F(wlg_wl_parameters, initialization_target_fraction);
    F(wlg_wl_parameters, initialization_temperature_fraction);
    F(wlg_wl_parameters, initialization_stall_attempts_per_spin);
    F(wlg_wl_parameters, initialization_temperature_multiplier);
    F(wlg_wl_parameters, initialization_max_temperature_fraction);
    F(wlg_wl_parameters, collect_window_statistics); F(wlg_wl_parameters, round_trip_margin_fraction);
    F(wlg_wl_parameters, nalivaiko_mod);
    S(wlg_run_config); F(wlg_run_config, emin); F(wlg_run_config, emax); F(wlg_run_config, bin_width);
    F(wlg_run_config, windows); F(wlg_run_config, walkers_per_window); F(wlg_run_config, overlap);
    F(wlg_run_config, explicit_windows); F(wlg_run_config, seed); F(wlg_run_config, wl);
    F(wlg_run_config, exchange_interval_attempts); F(wlg_run_config, max_attempts);
    F(wlg_run_config, checkpoint_interval_attempts); F(wlg_run_config, checkpoint_path);
    F(wlg_run_config, initial_spins); F(wlg_run_config, initial_spins_present);
    F(wlg_run_config, progress_interval_seconds); F(wlg_run_config, coupling_precision);
    F(wlg_run_config, recompute_interval_attempts);
    S(wlg_histogram_statistics); F(wlg_histogram_statistics, active_bins); F(wlg_histogram_statistics, covered_bins);
    F(wlg_histogram_statistics, minimum); F(wlg_histogram_statistics, mean); F(wlg_histogram_statistics, min_over_mean);
    F(wlg_histogram_statistics, coverage);
    S(wlg_walker_statistics); F(wlg_walker_statistics, walker_id); F(wlg_walker_statistics, window_id);
    F(wlg_walker_statistics, mpi_rank); F(wlg_walker_statistics, attempted); F(wlg_walker_statistics, accepted);
    F(wlg_walker_statistics, forced_accepted); F(wlg_walker_statistics, attempts_since_last_accepted);
    F(wlg_walker_statistics, energy); F(wlg_walker_statistics, factor); F(wlg_walker_statistics, active_bins);
    F(wlg_walker_statistics, minimum_histogram); F(wlg_walker_statistics, mean_histogram);
    F(wlg_walker_statistics, min_over_mean); F(wlg_walker_statistics, round_trips);
    S(wlg_run_totals); F(wlg_run_totals, attempted); F(wlg_run_totals, accepted); F(wlg_run_totals, forced_accepted);
    F(wlg_run_totals, exchange_attempted); F(wlg_run_totals, exchange_accepted); F(wlg_run_totals, converged);
    F(wlg_run_totals, epochs);
    S(wlg_epoch_timing); F(wlg_epoch_timing, epochs); F(wlg_epoch_timing, walk_ms); F(wlg_epoch_timing, exchange_ms);
    F(wlg_epoch_timing, total_ms); F(wlg_epoch_timing, attempted); F(wlg_epoch_timing, accepted);
    S(wlg_precision_report); F(wlg_precision_report, coupling_precision); F(wlg_precision_report, pad);
    F(wlg_precision_report, recompute_interval_attempts); F(wlg_precision_report, recomputes);
    F(wlg_precision_report, resynced); F(wlg_precision_report, deferred); F(wlg_precision_report, bin_changes);
    F(wlg_precision_report, max_field_drift); F(wlg_precision_report, max_energy_drift);
    S(wlg_autotune_report); F(wlg_autotune_report, walkers_per_block); F(wlg_autotune_report, epochs_per_graph);
    F(wlg_autotune_report, ms_per_epoch); F(wlg_autotune_report, trials); F(wlg_autotune_report, staging_ring); F(wlg_autotune_report, pad);
    S(wlg_fragment_view); F(wlg_fragment_view, window_begin); F(wlg_fragment_view, window_end);
    F(wlg_fragment_view, log_g); F(wlg_fragment_view, histogram); F(wlg_fragment_view, standard_error);
    F(wlg_fragment_view, valid);
    S(wlg_join_quality); F(wlg_join_quality, join_bin); F(wlg_join_quality, common_bins); F(wlg_join_quality, rmse);
    F(wlg_join_quality, max_abs_difference); F(wlg_join_quality, slope_difference);
    S(wlg_adaptive_parameters); F(wlg_adaptive_parameters, iterations); F(wlg_adaptive_parameters, pilot_mcs);
    F(wlg_adaptive_parameters, smoothing_width); F(wlg_adaptive_parameters, minimum_width);
    F(wlg_adaptive_parameters, diffusivity_floor_fraction); F(wlg_adaptive_parameters, curvature_weight);
    F(wlg_adaptive_parameters, round_trip_target); F(wlg_adaptive_parameters, maximum_round_trip_penalty);
    S(wlg_sampling_view); F(wlg_sampling_view, window_begin); F(wlg_sampling_view, window_end);
    F(wlg_sampling_view, squared_energy_displacement); F(wlg_sampling_view, displacement_samples);
    F(wlg_sampling_view, round_trips); F(wlg_sampling_view, walkers);
    S(wlg_snapshot); F(wlg_snapshot, walker_id); F(wlg_snapshot, spins); F(wlg_snapshot, fields);
    F(wlg_snapshot, energy); F(wlg_snapshot, log_g); F(wlg_snapshot, histogram); F(wlg_snapshot, active);
    F(wlg_snapshot, factor); F(wlg_snapshot, attempted); F(wlg_snapshot, accepted); F(wlg_snapshot, forced_accepted);
    F(wlg_snapshot, last_accepted_attempt); F(wlg_snapshot, stage); F(wlg_snapshot, rng_state);
    printf("\"end\": 0}\n");
    return 0;
}
