/*
 * wl_oracle.c — TEST INFRASTRUCTURE ONLY: plain-C restatement of the reference's REWL
 * hot path (Faikert/replica_exchange_wang_landau).  See wl_oracle.h for its role.
 *
 * It follows the reference operation for operation so that, given the same inputs, it
 * produces the same doubles: the same summation orders, no FMA contraction (the Makefile
 * builds it with -ffp-contract=off, as the reference's ISO C++20 build has none), glibc's
 * log() as the reference's std::log, and long double where the reference uses it.
 */
#include "wl_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_REPRESENTATIVES 9

static void set_err(char* err, size_t len, const char* fmt, ...) {
    if (!err || len == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

/* ---- xoshiro256** (include/wl/rng.hpp:10-56) ---------------------------------- */

typedef struct { uint64_t s[4]; } orc_rng;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* rng.hpp:46-51 */
static uint64_t splitmix(uint64_t* x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* rng.hpp:52-55 */
static void rng_seed(orc_rng* r, uint64_t seed, uint64_t stream) {
    uint64_t x = seed ^ (0xd2b74407b1ce6e93ULL * (stream + 1));
    for (int k = 0; k < 4; ++k) r->s[k] = splitmix(&x);
}

/* rng.hpp:16-23 */
static uint64_t rng_next(orc_rng* r) {
    uint64_t* s = r->s;
    const uint64_t result = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1];
    s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl64(s[3], 45);
    return result;
}

/* rng.hpp:25-27 */
static double rng_uniform(orc_rng* r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }

/* rng.hpp:29-36 */
static uint64_t rng_bounded(orc_rng* r, uint64_t bound) {
    if (bound == 0) return 0;
    const uint64_t threshold = (0 - bound) % bound;
    for (;;) {
        const uint64_t x = rng_next(r);
        if (x >= threshold) return x % bound;
    }
}

/* ---- physics (src/physics.cpp) ------------------------------------------------ */

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* physics.cpp:151-160 */
void orc_minimum_image(const double* d, const double* box, int periodic, double* out) {
    out[0] = d[0]; out[1] = d[1]; out[2] = d[2];
    if (!periodic) return;
    if (box[0] > 0.0) out[0] -= box[0] * nearbyint(out[0] / box[0]);
    if (box[1] > 0.0) out[1] -= box[1] * nearbyint(out[1] / box[1]);
    if (box[2] > 0.0) out[2] -= box[2] * nearbyint(out[2] / box[2]);
}

/* physics.cpp:162-170; returns 0 and sets *ok = 0 for coincident sites */
static double dipolar_pair_checked(const double* d, const double* ai, const double* aj, double scale,
                                   int* ok) {
    const double r2 = dot3(d, d);
    if (!(r2 > 0.0)) { *ok = 0; return 0.0; }
    const double inv_r = 1.0 / sqrt(r2);
    const double rhat[3] = {d[0] * inv_r, d[1] * inv_r, d[2] * inv_r};
    const double angular = dot3(ai, aj) - 3.0 * dot3(ai, rhat) * dot3(aj, rhat);
    return scale * angular * inv_r * inv_r * inv_r;
}

double orc_dipolar_pair(const double* d, const double* ai, const double* aj, double scale) {
    int ok = 1;
    const double v = dipolar_pair_checked(d, ai, aj, scale, &ok);
    return ok ? v : NAN;
}

struct orc_couplings {
    uint64_t n;
    int csr;
    double* dense;     /* n*n, row-major                                  */
    uint64_t* offsets; /* CSR: n+1                                       */
    uint64_t* columns; /* CSR: nnz                                       */
    double* values;    /* CSR: nnz                                       */
    int update_fp32;   /* add_flip_delta with FP32-rounded couplings      */
    int update_bf16;   /* add_flip_delta with BF16 couplings and row scale */
    double* bf16_value; /* dense, n*n: row k holds scale_k * bf16(J_kj / scale_k) */
};

/* Geometry::validate (physics.cpp:34-56) */
static int validate_system(const wlg_system* s, char* err, size_t len) {
    if (s->n == 0) { set_err(err, len, "Geometry contains no sites"); return WLG_ERR_INVALID_ARGUMENT; }
    if (s->periodic) {
        for (int k = 0; k < 3; ++k)
            if (!(isfinite(s->box[k]) && s->box[k] >= 0.0)) {
                set_err(err, len, "Periodic box lengths must be finite and non-negative");
                return WLG_ERR_INVALID_ARGUMENT;
            }
        if (s->box[0] == 0.0 && s->box[1] == 0.0 && s->box[2] == 0.0) {
            set_err(err, len, "At least one periodic box length must be positive");
            return WLG_ERR_INVALID_ARGUMENT;
        }
    }
    for (uint64_t i = 0; i < s->n; ++i) {
        const double* p = s->positions + 3 * i;
        if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) {
            set_err(err, len, "Site coordinates must be finite");
            return WLG_ERR_INVALID_ARGUMENT;
        }
        const double length = sqrt(dot3(s->axes + 3 * i, s->axes + 3 * i));
        if (fabs(length - 1.0) > 1e-10) {
            set_err(err, len, "Ising axes must be normalized");
            return WLG_ERR_INVALID_ARGUMENT;
        }
    }
    return 0;
}

/* pair_for (physics.cpp:26-30) with i < j */
static double pair_for(const wlg_system* s, uint64_t i, uint64_t j, int* ok, double* norm_out) {
    const double* pi = s->positions + 3 * i;
    const double* pj = s->positions + 3 * j;
    const double raw[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
    double d[3];
    orc_minimum_image(raw, s->box, s->periodic, d);
    if (norm_out) *norm_out = sqrt(dot3(d, d));
    return dipolar_pair_checked(d, s->axes + 3 * i, s->axes + 3 * j, s->coupling_scale, ok);
}

/* DenseCouplings ctor (physics.cpp:172-184) / CsrCouplings ctor (physics.cpp:197-223).
 * The CSR rows are filled in increasing column order, which is the order the reference's
 * sort by (row, column) produces. */
orc_couplings* orc_couplings_create(const wlg_system* s, char* err, size_t len) {
    if (validate_system(s, err, len)) return NULL;
    orc_couplings* c = calloc(1, sizeof *c);
    c->n = s->n;
    const uint64_t n = s->n;
    if (!(s->cutoff > 0.0)) {
        c->dense = calloc(n * n, sizeof(double));
        for (uint64_t i = 0; i < n; ++i)
            for (uint64_t j = i + 1; j < n; ++j) {
                int ok = 1;
                const double v = pair_for(s, i, j, &ok, NULL);
                if (!ok) { set_err(err, len, "Coincident dipole sites"); orc_couplings_destroy(c); return NULL; }
                c->dense[i * n + j] = v;
                c->dense[j * n + i] = v;
            }
        return c;
    }
    c->csr = 1;
    c->offsets = calloc(n + 1, sizeof(uint64_t));
    /* pass 1: count (every unordered pair evaluated once, in i<j orientation) */
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = i + 1; j < n; ++j) {
            int ok = 1;
            double r = 0.0;
            (void)pair_for(s, i, j, &ok, &r);
            if (r <= s->cutoff) {
                if (!ok) { set_err(err, len, "Coincident dipole sites"); orc_couplings_destroy(c); return NULL; }
                c->offsets[i + 1]++;
                c->offsets[j + 1]++;
            }
        }
    for (uint64_t i = 1; i <= n; ++i) c->offsets[i] += c->offsets[i - 1];
    const uint64_t nnz = c->offsets[n];
    c->columns = malloc((nnz ? nnz : 1) * sizeof(uint64_t));
    c->values = malloc((nnz ? nnz : 1) * sizeof(double));
    uint64_t* fill = malloc((n + 1) * sizeof(uint64_t));
    memcpy(fill, c->offsets, (n + 1) * sizeof(uint64_t));
    for (uint64_t row = 0; row < n; ++row)
        for (uint64_t col = 0; col < n; ++col) {
            if (col == row) continue;
            const uint64_t a = row < col ? row : col, b = row < col ? col : row;
            int ok = 1;
            double r = 0.0;
            const double v = pair_for(s, a, b, &ok, &r);
            if (r <= s->cutoff) {
                c->columns[fill[row]] = col;
                c->values[fill[row]] = v;
                fill[row]++;
            }
        }
    free(fill);
    return c;
}

void orc_couplings_destroy(orc_couplings* c) {
    if (!c) return;
    free(c->dense); free(c->offsets); free(c->columns); free(c->values); free(c->bf16_value);
    free(c);
}

uint64_t orc_couplings_size(const orc_couplings* c) { return c->n; }
uint64_t orc_couplings_nnz(const orc_couplings* c) { return c->csr ? c->offsets[c->n] : c->n * c->n; }

/* Couplings::at (physics.cpp:186-188, 225-229) as a dense matrix */
void orc_couplings_dense(const orc_couplings* c, double* out) {
    const uint64_t n = c->n;
    if (!c->csr) { memcpy(out, c->dense, n * n * sizeof(double)); return; }
    memset(out, 0, n * n * sizeof(double));
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t k = c->offsets[i]; k < c->offsets[i + 1]; ++k) out[i * n + c->columns[k]] = c->values[k];
}

/* local_fields (physics.cpp:238-251).  For CSR the reference also adds at(i,j)*s_j = +-0.0
 * for every non-neighbour j; starting from +0.0 those additions can never change the sum,
 * so only the neighbours, in column order, are added here. */
void orc_local_fields(const orc_couplings* c, const int8_t* spins, double* fields) {
    const uint64_t n = c->n;
    for (uint64_t i = 0; i < n; ++i) {
        double sum = 0.0;
        if (!c->csr) {
            for (uint64_t j = 0; j < n; ++j) sum += c->dense[i * n + j] * (double)spins[j];
        } else {
            for (uint64_t k = c->offsets[i]; k < c->offsets[i + 1]; ++k)
                sum += c->values[k] * (double)spins[c->columns[k]];
        }
        fields[i] = sum;
    }
}

/* total_energy (physics.cpp:253-259) */
double orc_total_energy(const orc_couplings* c, const int8_t* spins) {
    double* f = malloc(c->n * sizeof(double));
    orc_local_fields(c, spins, f);
    double energy = 0.0;
    for (uint64_t i = 0; i < c->n; ++i) energy += 0.5 * (double)spins[i] * f[i];
    free(f);
    return energy;
}

/* add_flip_delta (physics.cpp:190-195, 231-236) */
static double update_value(const orc_couplings* c, double v) { return c->update_fp32 ? (double)(float)v : v; }

static void add_flip_delta(const orc_couplings* c, uint64_t flipped, int8_t old_spin, double* fields) {
    const double multiplier = -2.0 * (double)old_spin;
    const uint64_t n = c->n;
    if (!c->csr && c->update_bf16) { /* the flipped site's BF16 row; every product is exact */
        const double* row = c->bf16_value + flipped * n;
        for (uint64_t j = 0; j < n; ++j) fields[j] += multiplier * row[j];
    } else if (!c->csr) {
        for (uint64_t j = 0; j < n; ++j) fields[j] += multiplier * update_value(c, c->dense[j * n + flipped]);
    } else {
        for (uint64_t k = c->offsets[flipped]; k < c->offsets[flipped + 1]; ++k)
            fields[c->columns[k]] += multiplier * update_value(c, c->values[k]);
    }
}

void orc_couplings_set_update_fp32(orc_couplings* c, int on) { c->update_fp32 = on != 0; }

/* Round to nearest even at bfloat16's 8 significant bits (subnormal spacing 2^-133), directly
 * from the double (one rounding, as the device's double-to-bf16 conversion does). */
double orc_bf16_round(double x) {
    if (x == 0.0 || !isfinite(x)) return x;
    int e = 0;
    (void)frexp(x, &e); /* |x| = m 2^e, 0.5 <= m < 1 */
    int q = e - 8;
    if (q < -133) q = -133;
    return ldexp(nearbyint(ldexp(x, -q)), q);
}

/* The engine's BF16 form of dense couplings: per row k the scale s_k = (float) max_j |J_kj|
 * (1 for a zero row) and the values bf16(J_kj / s_k); an accepted flip of site k adds
 * (-2 s) * s_k * bf16(J_kj / s_k) to field j, a product exact in FP64. */
void orc_couplings_set_update_bf16(orc_couplings* c, int on) {
    c->update_bf16 = on != 0 && !c->csr;
    if (!c->update_bf16 || c->bf16_value) return;
    const uint64_t n = c->n;
    c->bf16_value = malloc(n * n * sizeof(double));
    for (uint64_t k = 0; k < n; ++k) {
        double mx = 0.0;
        for (uint64_t j = 0; j < n; ++j) mx = fmax(mx, fabs(c->dense[k * n + j]));
        const float sc = mx > 0.0 ? (float)mx : 1.0f;
        for (uint64_t j = 0; j < n; ++j)
            c->bf16_value[k * n + j] = (double)sc * orc_bf16_round(c->dense[k * n + j] / (double)sc);
    }
}

void orc_couplings_csr(const orc_couplings* c, uint64_t* offsets, uint64_t* columns, double* values) {
    if (!c->csr) return;
    const uint64_t nnz = c->offsets[c->n];
    memcpy(offsets, c->offsets, (c->n + 1) * sizeof(uint64_t));
    memcpy(columns, c->columns, nnz * sizeof(uint64_t));
    memcpy(values, c->values, nnz * sizeof(double));
}

/* ---- energy grid and windows (src/wang_landau.cpp:13-61) ---------------------- */

/* EnergyGrid::validate (wang_landau.cpp:13-20) */
static int grid_validate(double mn, double mx, double w) {
    if (!isfinite(mn) || !isfinite(mx) || !isfinite(w) || !(mx > mn) || !(w > 0.0)) return 1;
    const double count = (mx - mn) / w;
    if (fabs(count - round(count)) > 1e-9 * fmax(1.0, count)) return 2;
    return 0;
}

int orc_grid_bins(double mn, double mx, double w, uint64_t* bins) {
    if (grid_validate(mn, mx, w)) return WLG_ERR_INVALID_ARGUMENT;
    *bins = (uint64_t)llround((mx - mn) / w);
    return 0;
}

/* EnergyGrid::index (wang_landau.cpp:27-34) */
int64_t orc_grid_index(double mn, double mx, double w, double e) {
    if (!isfinite(e) || e < mn || e > mx) return -1;
    uint64_t raw = (uint64_t)floor((e - mn) / w);
    const uint64_t count = (uint64_t)llround((mx - mn) / w);
    if (raw == count && e == mx) raw = count - 1;
    if (raw >= count) return -1;
    return (int64_t)raw;
}

/* partition_windows (wang_landau.cpp:40-61) */
int orc_partition_windows(uint64_t bins, uint64_t count, double overlap, uint64_t* out) {
    if (bins == 0 || count == 0 || count > bins || overlap < 0.0 || overlap >= 1.0) return WLG_ERR_INVALID_ARGUMENT;
    if (count == 1) { out[0] = 0; out[1] = bins; return 0; }
    const double denominator = 1.0 + (double)(count - 1) * (1.0 - overlap);
    uint64_t size = (uint64_t)ceil((double)bins / denominator);
    if (size > bins) size = bins;
    if (size < 2) size = 2;
    const uint64_t span = bins - size;
    for (uint64_t w = 0; w < count; ++w) {
        const uint64_t begin = (uint64_t)llround((double)(w * span) / (double)(count - 1));
        out[2 * w] = begin;
        out[2 * w + 1] = begin + size;
    }
    out[2 * count - 1] = bins;
    for (uint64_t w = 1; w < count; ++w)
        if (out[2 * w] >= out[2 * (w - 1) + 1]) return WLG_ERR_INVALID_ARGUMENT;
    return 0;
}

/* ---- the walker (src/wang_landau.cpp:63-510) ---------------------------------- */

struct orc_walker {
    uint64_t id;
    const orc_couplings* J;
    uint64_t n;
    double gmin, gmax, gw;
    uint64_t bins;
    uint64_t wb, we;
    wlg_wl_parameters p;
    orc_rng rng;
    int8_t* spins;
    double* fields;
    double energy;
    double* log_g;
    uint64_t* hist;
    uint8_t* active;
    uint8_t* refine;
    double* sqdisp;
    uint64_t* dsamples;
    uint64_t active_count, refine_count;
    double factor;
    uint64_t attempted, accepted, forced, last_acc;
    uint64_t time_offset; /* 1/t: f = active / (attempted + time_offset); 0: the reference's rule */
    int stage;
    uint8_t rt_state;
    uint64_t round_trips;
    double rep_target[ORC_REPRESENTATIVES], rep_dist[ORC_REPRESENTATIVES], rep_energy[ORC_REPRESENTATIVES];
    uint8_t rep_present[ORC_REPRESENTATIVES];
    int8_t* rep_spins;
};

static int64_t w_index(const orc_walker* w, double e) { return orc_grid_index(w->gmin, w->gmax, w->gw, e); }
static int w_contains(const orc_walker* w, int64_t b) { return b >= 0 && (uint64_t)b >= w->wb && (uint64_t)b < w->we; }

/* time_offset of a warm-started walker whose first covered check continues the schedule */
#define ORC_CONTINUE_SCHEDULE (~(uint64_t)0)

/* update_current_bin (wang_landau.cpp:290-303) */
static int update_current_bin(orc_walker* w, char* err, size_t len) {
    const int64_t b = w_index(w, w->energy);
    if (!w_contains(w, b)) { set_err(err, len, "Invalid current energy bin"); return WLG_ERR_RUNTIME; }
    ++w->hist[b];
    if (w->active[b] == 0) { w->active[b] = 1; ++w->active_count; }
    if (w->p.nalivaiko_mod && w->refine[b] == 0) { w->refine[b] = 1; ++w->refine_count; }
    if (w->stage != WLG_STAGE_FROZEN) w->log_g[b] += w->factor;
    return 0;
}

/* update_inverse_time_factor (wang_landau.cpp:309-315) */
static void update_inverse_time_factor(orc_walker* w) {
    if (w->stage != WLG_STAGE_INVERSE_TIME) return;
    const uint64_t count = w->active_count;
    if (count != 0 && w->attempted != 0) w->factor = (double)count / (double)(w->attempted + w->time_offset);
    if (w->factor <= w->p.final_factor) w->stage = WLG_STAGE_FROZEN;
}

static double w_lower(const orc_walker* w) { return w->gmin + (double)w->wb * w->gw; }
static double w_upper(const orc_walker* w) { return w->gmin + (double)w->we * w->gw; }

/* update_round_trip_state (wang_landau.cpp:317-330) */
static void update_round_trip_state(orc_walker* w) {
    if (!w->p.collect_window_statistics) return;
    const double lower = w_lower(w), upper = w_upper(w);
    const double margin = w->p.round_trip_margin_fraction * (upper - lower);
    if (w->energy <= lower + margin) {
        if (w->rt_state == 2) { ++w->round_trips; w->rt_state = 1; }
        else if (w->rt_state == 0) w->rt_state = 1;
    } else if (w->energy >= upper - margin && w->rt_state == 1) {
        w->rt_state = 2;
    }
}

/* update_representatives (wang_landau.cpp:332-342) */
static void update_representatives(orc_walker* w) {
    if (!w->p.collect_window_statistics) return;
    for (int r = 0; r < ORC_REPRESENTATIVES; ++r) {
        const double distance = fabs(w->energy - w->rep_target[r]);
        if (distance < w->rep_dist[r]) {
            w->rep_dist[r] = distance;
            w->rep_energy[r] = w->energy;
            memcpy(w->rep_spins + (uint64_t)r * w->n, w->spins, w->n);
            w->rep_present[r] = 1;
        }
    }
}

void orc_walker_destroy(orc_walker* w) {
    if (!w) return;
    free(w->spins); free(w->fields); free(w->log_g); free(w->hist); free(w->active); free(w->refine);
    free(w->sqdisp); free(w->dsamples); free(w->rep_spins);
    free(w);
}

static int params_valid(const wlg_wl_parameters* p) {
    return (p->flatness > 0.0 && p->flatness <= 1.0) && (p->final_factor > 0.0) &&
           p->check_interval_attempts != 0 && p->initialization_max_attempts != 0 &&
           (p->initialization_target_fraction > 0.0 && p->initialization_target_fraction <= 1.0) &&
           isfinite(p->initialization_temperature_fraction) && (p->initialization_temperature_fraction > 0.0) &&
           p->initialization_stall_attempts_per_spin != 0 &&
           isfinite(p->initialization_temperature_multiplier) &&
           (p->initialization_temperature_multiplier > 1.0) &&
           isfinite(p->initialization_max_temperature_fraction) &&
           !(p->initialization_max_temperature_fraction < p->initialization_temperature_fraction) &&
           isfinite(p->round_trip_margin_fraction) && !(p->round_trip_margin_fraction < 0.0) &&
           !(p->round_trip_margin_fraction >= 0.5);
}

static void finish_init(orc_walker* w, char* err, size_t len, int* status) {
    *status = update_current_bin(w, err, len);
    update_round_trip_state(w);
    update_representatives(w);
}

/* WangLandauWalker ctor (wang_landau.cpp:63-242), including the adaptive target-Metropolis
 * search and its failure message. */
orc_walker* orc_walker_create(const orc_couplings* c, uint64_t id, double emin, double emax, double width,
                              uint64_t window_begin, uint64_t window_end, const wlg_wl_parameters* p,
                              uint64_t seed, const int8_t* initial_spins, char* err, size_t len) {
    if (grid_validate(emin, emax, width)) { set_err(err, len, "Invalid energy grid"); return NULL; }
    uint64_t bins = 0;
    orc_grid_bins(emin, emax, width, &bins);
    if (window_begin >= window_end || window_end > bins) { set_err(err, len, "Invalid walker energy window"); return NULL; }
    if (!params_valid(p)) { set_err(err, len, "Invalid WL parameters"); return NULL; }
    const uint64_t n = c->n;
    if (initial_spins)
        for (uint64_t i = 0; i < n; ++i)
            if (initial_spins[i] != -1 && initial_spins[i] != 1) { set_err(err, len, "Spins must be +/-1"); return NULL; }
    orc_walker* w = calloc(1, sizeof *w);
    w->id = id; w->J = c; w->n = n;
    w->gmin = emin; w->gmax = emax; w->gw = width; w->bins = bins;
    w->wb = window_begin; w->we = window_end;
    w->p = *p;
    rng_seed(&w->rng, seed, id);
    w->spins = malloc(n);
    if (initial_spins) memcpy(w->spins, initial_spins, n); else memset(w->spins, 1, n);
    w->fields = malloc(n * sizeof(double));
    orc_local_fields(c, w->spins, w->fields);
    w->energy = orc_total_energy(c, w->spins);
    w->log_g = calloc(bins, sizeof(double));
    w->hist = calloc(bins, sizeof(uint64_t));
    w->active = calloc(bins, 1);
    w->refine = calloc(bins, 1);
    w->factor = 1.0;
    w->stage = WLG_STAGE_WANG_LANDAU;
    if (p->collect_window_statistics) {
        w->sqdisp = calloc(bins, sizeof(double));
        w->dsamples = calloc(bins, sizeof(uint64_t));
        const double lower = emin + (double)window_begin * width;
        const double upper = emin + (double)window_end * width;
        w->rep_target[0] = lower;
        for (int r = 1; r < ORC_REPRESENTATIVES; ++r)
            w->rep_target[r] = lower + (upper - lower) * ((double)r - 0.5) / (double)(ORC_REPRESENTATIVES - 1);
        for (int r = 0; r < ORC_REPRESENTATIVES; ++r) w->rep_dist[r] = INFINITY;
        w->rep_spins = calloc((uint64_t)ORC_REPRESENTATIVES * n, 1);
    }
    int status = 0;
    const int supplied = initial_spins != NULL;
    const int64_t initial_bin = w_index(w, w->energy);
    if (supplied && w_contains(w, initial_bin)) {
        finish_init(w, err, len, &status);
        if (status) { orc_walker_destroy(w); return NULL; }
        return w;
    }
    const double lower = w_lower(w), upper = w_upper(w);
    const double span = upper - lower;
    const double target = 0.5 * (lower + upper);
    const double target_fraction = supplied ? 1.0 : p->initialization_target_fraction;
    const double target_half_width = 0.5 * target_fraction * span;
    const double initial_T = fmax(width, p->initialization_temperature_fraction * span);
    const double maximum_T = fmax(initial_T, p->initialization_max_temperature_fraction * span);
    double T = initial_T;
    const uint64_t maximum_count = UINT64_MAX;
    const uint64_t stall = p->initialization_stall_attempts_per_spin > maximum_count / n
                               ? maximum_count
                               : p->initialization_stall_attempts_per_spin * n;
    uint64_t since = 0, increases = 0, restarts = 0;
    double highest_T = T;
    double min_reached = w->energy, max_reached = w->energy, closest = w->energy;
    double closest_distance = fabs(w->energy - target);
#define RECORD(candidate, improved_out)                                         \
    do {                                                                        \
        const double cand_ = (candidate);                                       \
        min_reached = (cand_ < min_reached) ? cand_ : min_reached;              \
        max_reached = (max_reached < cand_) ? cand_ : max_reached;              \
        const double dist_ = fabs(cand_ - target);                              \
        (improved_out) = 0;                                                     \
        if (dist_ < closest_distance) { closest_distance = dist_; closest = cand_; (improved_out) = 1; } \
    } while (0)
#define IN_BAND(e) (w_contains(w, w_index(w, (e))) && fabs((e) - target) <= target_half_width)
    for (uint64_t step = 0; step < p->initialization_max_attempts; ++step) {
        if (IN_BAND(w->energy)) {
            finish_init(w, err, len, &status);
            if (status) { orc_walker_destroy(w); return NULL; }
            return w;
        }
        if (since >= stall) {
            if (T < maximum_T) {
                T = fmin(maximum_T, T * p->initialization_temperature_multiplier);
                highest_T = fmax(highest_T, T);
                ++increases;
            } else {
                for (uint64_t i = 0; i < n; ++i) w->spins[i] = rng_bounded(&w->rng, 2) == 0 ? -1 : 1;
                orc_local_fields(c, w->spins, w->fields);
                w->energy = orc_total_energy(c, w->spins);
                int unused;
                RECORD(w->energy, unused);
                (void)unused;
                T = initial_T;
                ++restarts;
            }
            since = 0;
            if (IN_BAND(w->energy)) {
                finish_init(w, err, len, &status);
                if (status) { orc_walker_destroy(w); return NULL; }
                return w;
            }
        }
        const uint64_t i = rng_bounded(&w->rng, n);
        const int8_t old = w->spins[i];
        const double delta = -2.0 * (double)w->spins[i] * w->fields[i];
        const double proposed = w->energy + delta;
        const double log_acceptance = (fabs(w->energy - target) - fabs(proposed - target)) / T;
        int improved = 0;
        if (log_acceptance >= 0.0 || log(fmax(rng_uniform(&w->rng), 0x1.0p-53)) < log_acceptance) {
            add_flip_delta(c, i, old, w->fields);
            w->spins[i] = (int8_t)-old;
            w->energy = proposed;
            RECORD(w->energy, improved);
        }
        if (improved) since = 0;
        else if (since < maximum_count) ++since;
    }
    if (IN_BAND(w->energy)) {
        finish_init(w, err, len, &status);
        if (status) { orc_walker_destroy(w); return NULL; }
        return w;
    }
#undef IN_BAND
#undef RECORD
    {
        char bin_text[64];
        const int64_t cb = w_index(w, closest);
        if (cb >= 0) snprintf(bin_text, sizeof bin_text, " (bin %lld)", (long long)cb);
        else snprintf(bin_text, sizeof bin_text, " (outside the energy grid)");
        set_err(err, len,
                "Target Metropolis initialization did not reach target band [%.17g, %.17g] for energy "
                "window bins [%llu, %llu), energy bounds [%.17g, %.17g%c after %llu attempts; reached "
                "energy range [%.17g, %.17g], closest energy %.17g%s, distance to target band %.17g; "
                "adaptive search used %llu temperature increases up to %.17g and %llu random restarts "
                "(stall interval %llu attempts)",
                target - target_half_width, target + target_half_width, (unsigned long long)w->wb,
                (unsigned long long)w->we, lower, upper, w->we == bins ? ']' : ')',
                (unsigned long long)p->initialization_max_attempts, min_reached, max_reached, closest, bin_text,
                fmax(0.0, closest_distance - target_half_width), (unsigned long long)increases, highest_T,
                (unsigned long long)restarts, (unsigned long long)stall);
    }
    orc_walker_destroy(w);
    return NULL;
}

/* attempt_flip (wang_landau.cpp:244-284) */
int orc_walker_attempt(orc_walker* w, int* accepted_out, char* err, size_t len) {
    const uint64_t i = rng_bounded(&w->rng, w->n);
    const int64_t old_bin = w_index(w, w->energy);
    if (!w_contains(w, old_bin)) { set_err(err, len, "Walker escaped its energy window"); return WLG_ERR_ESCAPED; }
    const int8_t old_spin = w->spins[i];
    const double delta = -2.0 * (double)w->spins[i] * w->fields[i];
    const double proposed = w->energy + delta;
    const int64_t new_bin = w_index(w, proposed);
    int accepted = 0, forced = 0;
    if (w_contains(w, new_bin)) {
        const double log_ratio = w->log_g[old_bin] - w->log_g[new_bin];
        const int force_due = w->p.force_accept_after_attempts != 0 &&
                              w->attempted - w->last_acc >= w->p.force_accept_after_attempts;
        if (log_ratio >= 0.0) accepted = 1;
        else if (force_due) accepted = forced = 1;
        else accepted = log(fmax(rng_uniform(&w->rng), 0x1.0p-53)) < log_ratio;
    }
    ++w->attempted;
    if (accepted) {
        add_flip_delta(w->J, i, old_spin, w->fields);
        w->spins[i] = (int8_t)-old_spin;
        w->energy = proposed;
        ++w->accepted;
        if (forced) ++w->forced;
        w->last_acc = w->attempted;
    }
    if (w->p.collect_window_statistics) {
        const double displacement = accepted ? delta : 0.0;
        w->sqdisp[old_bin] += displacement * displacement;
        ++w->dsamples[old_bin];
    }
    update_inverse_time_factor(w);
    const int status = update_current_bin(w, err, len);
    if (status) return status;
    if (accepted) { update_round_trip_state(w); update_representatives(w); }
    if (accepted_out) *accepted_out = accepted;
    return 0;
}

/* run_attempts (wang_landau.cpp:286-288) */
int orc_walker_run(orc_walker* w, uint64_t count, char* err, size_t len) {
    for (uint64_t k = 0; k < count; ++k) {
        const int s = orc_walker_attempt(w, NULL, err, len);
        if (s) return s;
    }
    return 0;
}

/* histogram_statistics (wang_landau.cpp:344-367) */
void orc_walker_histogram_statistics(const orc_walker* w, wlg_histogram_statistics* st) {
    const uint8_t* mask = w->p.nalivaiko_mod ? w->refine : w->active;
    memset(st, 0, sizeof *st);
    st->active_bins = w->p.nalivaiko_mod ? w->refine_count : w->active_count;
    long double total = 0.0L;
    st->minimum = UINT64_MAX;
    for (uint64_t i = w->wb; i < w->we; ++i) {
        if (!mask[i]) continue;
        if (w->hist[i] != 0) ++st->covered_bins;
        if (w->hist[i] < st->minimum) st->minimum = w->hist[i];
        total += (long double)w->hist[i];
    }
    if (st->active_bins == 0) { st->minimum = 0; return; }
    st->mean = (double)(total / (long double)st->active_bins);
    st->min_over_mean = st->mean > 0.0 ? (double)st->minimum / st->mean : 0.0;
    st->coverage = (double)st->covered_bins / (double)st->active_bins;
}

/* flat / covered / ready_for_iteration (wang_landau.cpp:369-387) */
static int w_flat(const orc_walker* w) {
    if (w->stage != WLG_STAGE_WANG_LANDAU) return 1;
    wlg_histogram_statistics s;
    orc_walker_histogram_statistics(w, &s);
    return s.active_bins != 0 && s.minimum >= w->p.minimum_visits && s.min_over_mean >= w->p.flatness;
}
static int w_covered(const orc_walker* w) {
    if (w->stage != WLG_STAGE_WANG_LANDAU) return 1;
    wlg_histogram_statistics s;
    orc_walker_histogram_statistics(w, &s);
    return s.active_bins != 0 && s.covered_bins == s.active_bins;
}
static int w_ready(const orc_walker* w) {
    return w->stage == WLG_STAGE_WANG_LANDAU && (w->p.inverse_time_enabled ? w_covered(w) : w_flat(w));
}
void orc_walker_flags(const orc_walker* w, int* flat, int* covered, int* ready) {
    *flat = w_flat(w); *covered = w_covered(w); *ready = w_ready(w);
}

/* begin_next_iteration + freeze_if_finished (wang_landau.cpp:389-413) */
int orc_walker_begin_next_iteration(orc_walker* w, char* err, size_t len) {
    if (!w_ready(w)) { set_err(err, len, "WL iteration is not complete"); return WLG_ERR_LOGIC; }
    w->factor *= 0.5;
    for (uint64_t i = w->wb; i < w->we; ++i) w->hist[i] = 0;
    if (w->p.nalivaiko_mod) {
        for (uint64_t i = w->wb; i < w->we; ++i) w->refine[i] = 0;
        w->refine_count = 0;
    }
    if (w->p.inverse_time_enabled) {
        if (w->time_offset == ORC_CONTINUE_SCHEDULE) {
            /* warm start continuing the schedule: 1/t from the factor reached, as if
             * round(active / factor) attempts had been made */
            const double made = fmin(nearbyint((double)w->active_count / w->factor), 0x1.0p62);
            const double attempted = (double)w->attempted;
            w->time_offset = made > attempted ? (uint64_t)(made - attempted) : 0;
            w->stage = WLG_STAGE_INVERSE_TIME;
        } else {
            const double inverse_time =
                w->attempted == 0 ? 1.0 : (double)w->active_count / (double)(w->attempted + w->time_offset);
            if (w->factor <= inverse_time) { w->stage = WLG_STAGE_INVERSE_TIME; w->factor = inverse_time; }
        }
    }
    if (w->factor <= w->p.final_factor) w->stage = WLG_STAGE_FROZEN;
    return 0;
}

/* snapshot (wang_landau.cpp:415-418) */
void orc_walker_snapshot(const orc_walker* w, wlg_snapshot* s) {
    s->walker_id = w->id;
    if (s->spins) memcpy(s->spins, w->spins, w->n);
    if (s->fields) memcpy(s->fields, w->fields, w->n * sizeof(double));
    s->energy = w->energy;
    if (s->log_g) memcpy(s->log_g, w->log_g, w->bins * sizeof(double));
    if (s->histogram) memcpy(s->histogram, w->hist, w->bins * sizeof(uint64_t));
    if (s->active) memcpy(s->active, w->active, w->bins);
    s->factor = w->factor;
    s->attempted = w->attempted;
    s->accepted = w->accepted;
    s->forced_accepted = w->forced;
    s->last_accepted_attempt = w->last_acc;
    s->stage = (uint8_t)w->stage;
    memcpy(s->rng_state, w->rng.s, sizeof w->rng.s);
}

/* restore (wang_landau.cpp:420-466) */
int orc_walker_restore(orc_walker* w, const wlg_snapshot* s, char* err, size_t len) {
    if (s->walker_id != w->id) { set_err(err, len, "Checkpoint is incompatible with walker"); return WLG_ERR_INVALID_ARGUMENT; }
    if (s->last_accepted_attempt > s->attempted) {
        set_err(err, len, "Checkpoint has an invalid last accepted attempt");
        return WLG_ERR_INVALID_ARGUMENT;
    }
    if (s->forced_accepted > s->accepted) {
        set_err(err, len, "Checkpoint has an invalid forced acceptance count");
        return WLG_ERR_INVALID_ARGUMENT;
    }
    if (!w->p.inverse_time_enabled && s->stage == WLG_STAGE_INVERSE_TIME) {
        set_err(err, len, "Checkpoint uses disabled inverse-time refinement");
        return WLG_ERR_INVALID_ARGUMENT;
    }
    memcpy(w->spins, s->spins, w->n);
    memcpy(w->fields, s->fields, w->n * sizeof(double));
    w->energy = s->energy;
    memcpy(w->log_g, s->log_g, w->bins * sizeof(double));
    memcpy(w->hist, s->histogram, w->bins * sizeof(uint64_t));
    memcpy(w->active, s->active, w->bins);
    w->factor = s->factor;
    w->attempted = s->attempted;
    w->accepted = s->accepted;
    w->active_count = 0;
    memset(w->refine, 0, w->bins);
    w->refine_count = 0;
    for (uint64_t i = w->wb; i < w->we; ++i) {
        w->active[i] = w->active[i] != 0 ? 1 : 0;
        w->active_count += w->active[i];
        if (w->p.nalivaiko_mod) {
            w->refine[i] = (uint8_t)(w->hist[i] != 0);
            w->refine_count += w->refine[i];
        }
    }
    w->forced = s->forced_accepted;
    w->last_acc = s->last_accepted_attempt;
    w->stage = s->stage;
    memcpy(w->rng.s, s->rng_state, sizeof w->rng.s);
    if (w->p.collect_window_statistics) {
        memset(w->sqdisp, 0, w->bins * sizeof(double));
        memset(w->dsamples, 0, w->bins * sizeof(uint64_t));
        w->rt_state = 0;
        w->round_trips = 0;
        update_round_trip_state(w);
        for (int r = 0; r < ORC_REPRESENTATIVES; ++r) { w->rep_dist[r] = INFINITY; w->rep_present[r] = 0; }
        update_representatives(w);
    }
    const double exact = orc_total_energy(w->J, w->spins);
    if (fabs(exact - w->energy) > 1e-9 * fmax(1.0, fabs(exact))) {
        set_err(err, len, "Checkpoint energy does not match spin configuration");
        return WLG_ERR_RUNTIME;
    }
    double* exact_fields = malloc(w->n * sizeof(double));
    orc_local_fields(w->J, w->spins, exact_fields);
    for (uint64_t i = 0; i < w->n; ++i)
        if (fabs(exact_fields[i] - w->fields[i]) > 1e-9 * fmax(1.0, fabs(exact_fields[i]))) {
            free(exact_fields);
            set_err(err, len, "Checkpoint local fields do not match spin configuration");
            return WLG_ERR_RUNTIME;
        }
    free(exact_fields);
    return 0;
}

/* exchange_log_probability (wang_landau.cpp:497-508) */
double orc_walker_exchange_log_probability(const orc_walker* a, const orc_walker* b) {
    const int64_t x_here = w_index(a, a->energy), y_here = w_index(a, b->energy);
    const int64_t x_there = w_index(b, a->energy), y_there = w_index(b, b->energy);
    if (!w_contains(a, x_here) || !w_contains(a, y_here) || !w_contains(b, x_there) || !w_contains(b, y_there))
        return -INFINITY;
    return a->log_g[x_here] - a->log_g[y_here] + b->log_g[y_there] - b->log_g[x_there];
}

/* swap_configuration (wang_landau.cpp:483-495) */
int orc_walker_swap(orc_walker* a, orc_walker* b, char* err, size_t len) {
    const int64_t this_bin = w_index(a, b->energy), other_bin = w_index(b, a->energy);
    if (!w_contains(a, this_bin) || !w_contains(b, other_bin)) {
        set_err(err, len, "Replica exchange would violate an energy window");
        return WLG_ERR_INVALID_ARGUMENT;
    }
    int8_t* sp = a->spins; a->spins = b->spins; b->spins = sp;
    double* f = a->fields; a->fields = b->fields; b->fields = f;
    const double e = a->energy; a->energy = b->energy; b->energy = e;
    update_round_trip_state(a);
    update_round_trip_state(b);
    update_representatives(a);
    update_representatives(b);
    return 0;
}

void orc_walker_counters(const orc_walker* w, uint64_t* out) {
    out[0] = w->attempted; out[1] = w->accepted; out[2] = w->forced; out[3] = w->last_acc;
}

void orc_walker_pilot(const orc_walker* w, double* sq, uint64_t* samples, uint64_t* round_trips,
                      double* rep_energies, int8_t* rep_spins, uint8_t* rep_present) {
    if (w->p.collect_window_statistics) {
        if (sq) memcpy(sq, w->sqdisp, w->bins * sizeof(double));
        if (samples) memcpy(samples, w->dsamples, w->bins * sizeof(uint64_t));
    }
    *round_trips = w->round_trips;
    if (!w->p.collect_window_statistics) return;
    for (int r = 0; r < ORC_REPRESENTATIVES; ++r) {
        rep_energies[r] = w->rep_energy[r];
        rep_present[r] = w->rep_present[r];
        if (w->rep_present[r]) memcpy(rep_spins + (uint64_t)r * w->n, w->rep_spins + (uint64_t)r * w->n, w->n);
    }
}

/* ---- checkpoint format (src/io.cpp:539-572) ----------------------------------- */

static int write_vec(FILE* f, const void* data, uint64_t count, size_t elem) {
    return fwrite(&count, 8, 1, f) == 1 && (count == 0 || fwrite(data, elem, count, f) == count);
}

static int save_checkpoint(const char* path, const orc_walker* w) {
    char tmp[4096];
    snprintf(tmp, sizeof tmp, "%s.tmp", path);
    FILE* f = fopen(tmp, "wb");
    if (!f) return WLG_ERR_IO;
    const char magic[8] = {'W', 'L', 'C', 'H', 'K', 'P', '3', '\0'};
    int ok = fwrite(magic, 1, 8, f) == 8 && fwrite(&w->id, 8, 1, f) == 1;
    ok = ok && write_vec(f, w->spins, w->n, 1) && write_vec(f, w->fields, w->n, 8) && fwrite(&w->energy, 8, 1, f) == 1;
    ok = ok && write_vec(f, w->log_g, w->bins, 8) && write_vec(f, w->hist, w->bins, 8) && write_vec(f, w->active, w->bins, 1);
    const uint8_t stage = (uint8_t)w->stage;
    ok = ok && fwrite(&w->factor, 8, 1, f) == 1 && fwrite(&w->attempted, 8, 1, f) == 1 &&
         fwrite(&w->accepted, 8, 1, f) == 1 && fwrite(&w->forced, 8, 1, f) == 1 &&
         fwrite(&w->last_acc, 8, 1, f) == 1 && fwrite(&stage, 1, 1, f) == 1 && fwrite(w->rng.s, 8, 4, f) == 4;
    ok = (fclose(f) == 0) && ok;
    if (!ok) return WLG_ERR_IO;
    remove(path);
    return rename(tmp, path) == 0 ? 0 : WLG_ERR_IO;
}

static int read_exact(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

static int load_checkpoint_into(const char* path, const orc_walker* w, wlg_snapshot* s, int8_t* spins,
                                double* fields, double* log_g, uint64_t* hist, uint8_t* active) {
    FILE* f = fopen(path, "rb");
    if (!f) return WLG_ERR_IO;
    char magic[8];
    int ok = read_exact(f, magic, 8);
    int version = 0;
    if (ok && memcmp(magic, "WLCHKP1", 7) == 0) version = 1;
    if (ok && memcmp(magic, "WLCHKP2", 7) == 0) version = 2;
    if (ok && memcmp(magic, "WLCHKP3", 7) == 0) version = 3;
    if (!version) { fclose(f); return WLG_ERR_RUNTIME; }
    uint64_t count = 0;
    ok = read_exact(f, &s->walker_id, 8);
#define VEC(ptr, elem, expect)                                                          \
    ok = ok && read_exact(f, &count, 8) && count == (expect) && read_exact(f, (ptr), (size_t)(count * (elem)));
    VEC(spins, 1, w->n)
    VEC(fields, 8, w->n)
    ok = ok && read_exact(f, &s->energy, 8);
    VEC(log_g, 8, w->bins)
    VEC(hist, 8, w->bins)
    VEC(active, 1, w->bins)
#undef VEC
    ok = ok && read_exact(f, &s->factor, 8) && read_exact(f, &s->attempted, 8) && read_exact(f, &s->accepted, 8);
    s->forced_accepted = 0;
    if (version == 3) ok = ok && read_exact(f, &s->forced_accepted, 8);
    if (version >= 2) ok = ok && read_exact(f, &s->last_accepted_attempt, 8);
    else s->last_accepted_attempt = s->accepted == 0 ? 0 : s->attempted;
    ok = ok && read_exact(f, &s->stage, 1) && read_exact(f, s->rng_state, 32);
    fclose(f);
    s->spins = spins; s->fields = fields; s->log_g = log_g; s->histogram = hist; s->active = active;
    return ok ? 0 : WLG_ERR_RUNTIME;
}

/* ---- run_rewl, serial path (src/parallel.cpp:23-78, 157-166, 276-580) --------- */

struct orc_result {
    wlg_run_totals totals;
    uint64_t windows, bins, n;
    double* log_g;        /* windows x bins */
    uint64_t* histogram;  /* windows x bins */
    double* sem;          /* windows x bins */
    uint8_t* valid;       /* windows x bins */
    int collect;
    double* sq;           /* windows x bins */
    uint64_t* samples;    /* windows x bins */
    uint64_t* round_trips;/* windows */
    uint64_t* walker_counts;
    wlg_walker_statistics* stats;
    uint64_t stat_count;
    double* rep_energy;
    int8_t* rep_spins;
    uint64_t rep_count;
};

void orc_result_destroy(orc_result* r) {
    if (!r) return;
    free(r->log_g); free(r->histogram); free(r->sem); free(r->valid); free(r->sq); free(r->samples);
    free(r->round_trips); free(r->walker_counts); free(r->stats); free(r->rep_energy); free(r->rep_spins);
    free(r);
}

/* local_exchange (parallel.cpp:157-166) */
static int local_exchange(orc_walker* left, orc_walker* right, uint64_t seed, uint64_t epoch, uint64_t boundary,
                          int* swapped, char* err, size_t len) {
    const double logp = orc_walker_exchange_log_probability(left, right);
    orc_rng rng;
    rng_seed(&rng, seed ^ (epoch * 0x9e3779b97f4a7c15ULL), boundary);
    *swapped = 0;
    if (isfinite(logp) && (logp >= 0.0 || log(fmax(rng_uniform(&rng), 0x1.0p-53)) < logp)) {
        const int s = orc_walker_swap(left, right, err, len);
        if (s) return s;
        *swapped = 1;
    }
    return 0;
}

/* summarize_impl (parallel.cpp:23-62) */
static int summarize(orc_walker** ws, uint64_t count, uint64_t wb, uint64_t we, uint64_t bins, int allow_empty,
                     double* log_g, uint64_t* hist, double* sem, uint8_t* valid, char* err, size_t len) {
    for (uint64_t i = 0; i < bins; ++i) { log_g[i] = NAN; hist[i] = 0; sem[i] = NAN; valid[i] = 0; }
    for (uint64_t i = wb; i < we; ++i) {
        int v = 1;
        for (uint64_t k = 0; k < count; ++k) {
            v = v && ws[k]->active[i] != 0;
            hist[i] += ws[k]->hist[i];
        }
        valid[i] = v ? 1 : 0;
    }
    uint64_t ref = we;
    for (uint64_t i = wb; i < we; ++i) if (valid[i] == 1) { ref = i; break; }
    if (ref == we && allow_empty) return 0;
    if (ref == we) { set_err(err, len, "Walkers in an energy window have no common active bin"); return WLG_ERR_RUNTIME; }
    for (uint64_t i = wb; i < we; ++i) {
        if (valid[i] == 0) continue;
        log_g[i] = 0.0;
        for (uint64_t k = 0; k < count; ++k) log_g[i] += ws[k]->log_g[i] - ws[k]->log_g[ref];
        log_g[i] /= (double)count;
        if (count > 1) {
            double sd = 0.0;
            for (uint64_t k = 0; k < count; ++k) {
                const double value = ws[k]->log_g[i] - ws[k]->log_g[ref];
                const double delta = value - log_g[i];
                sd += delta * delta;
            }
            sem[i] = sqrt(sd / ((double)count * (double)(count - 1)));
        }
    }
    return 0;
}

/* RunConfig::validate (io.cpp:243-268), the part run_rewl exercises */
static int validate_config(const wlg_run_config* c, uint64_t bins_checked, char* err, size_t len) {
    (void)bins_checked;
    if (!isfinite(c->progress_interval_seconds) || c->progress_interval_seconds < 0.0 || c->windows == 0 ||
        c->walkers_per_window == 0 || c->overlap < 0.0 || c->overlap >= 1.0 || c->exchange_interval_attempts == 0 ||
        c->wl.check_interval_attempts == 0 || c->checkpoint_interval_attempts == 0 ||
        !isfinite(c->wl.round_trip_margin_fraction) || c->wl.round_trip_margin_fraction < 0.0 ||
        c->wl.round_trip_margin_fraction >= 0.5) {
        set_err(err, len, "Invalid run configuration");
        return WLG_ERR_INVALID_ARGUMENT;
    }
    if (grid_validate(c->emin, c->emax, c->bin_width)) {
        set_err(err, len, grid_validate(c->emin, c->emax, c->bin_width) == 1
                              ? "Invalid energy grid" : "Energy range must be an integer multiple of bin width");
        return WLG_ERR_INVALID_ARGUMENT;
    }
    uint64_t bins = 0;
    orc_grid_bins(c->emin, c->emax, c->bin_width, &bins);
    if (c->windows > bins) { set_err(err, len, "More windows than energy bins"); return WLG_ERR_INVALID_ARGUMENT; }
    if (c->explicit_windows) {
        const uint64_t* e = c->explicit_windows;
        if (e[0] != 0 || e[2 * c->windows - 1] != bins) {
            set_err(err, len, "Explicit energy windows must match the configured range");
            return WLG_ERR_INVALID_ARGUMENT;
        }
        for (uint64_t i = 0; i < c->windows; ++i)
            if (e[2 * i] >= e[2 * i + 1] || e[2 * i + 1] > bins ||
                (i != 0 && (e[2 * i] <= e[2 * (i - 1)] || e[2 * i] >= e[2 * (i - 1) + 1]))) {
                set_err(err, len, "Explicit energy windows must be ordered and overlap");
                return WLG_ERR_INVALID_ARGUMENT;
            }
    }
    return 0;
}

/* The engine's FP32- and BF16-couplings forms (extensions; the reference stores J in FP64
 * only): walkers are constructed from the FP64 couplings, then every accepted flip adds the
 * FP32-rounded coupling (update_value) or the BF16 row value times its row scale
 * (orc_couplings_set_update_bf16), and every R = ceil(recompute interval / exchange interval) epochs,
 * after the epoch's exchange and unless the run has just terminated, every walker's fields and
 * energy are recomputed from the FP64 couplings in the reference's order (local_fields,
 * total_energy) and replace the drifted ones, unless the recomputed energy lies outside the
 * walker's window (the resync is then deferred). */
static int check_precision(const wlg_run_config* cfg, char* err, size_t len) {
    if (cfg->coupling_precision == WLG_PRECISION_FP64 || cfg->coupling_precision == WLG_PRECISION_FP32 ||
        cfg->coupling_precision == WLG_PRECISION_BF16)
        return 0;
    set_err(err, len, "Unknown coupling precision");
    return 1;
}

static void recompute_fp64(orc_walker* const* ws, uint64_t total, const orc_couplings* c) {
    double* f64 = malloc(c->n * sizeof(double));
    for (uint64_t q = 0; q < total; ++q) {
        orc_walker* w = ws[q];
        orc_local_fields(c, w->spins, f64);
        const double e64 = orc_total_energy(c, w->spins);
        if (!w_contains(w, w_index(w, e64))) continue; /* deferred */
        memcpy(w->fields, f64, c->n * sizeof(double));
        w->energy = e64;
    }
    free(f64);
}

void orc_walker_warm_start(orc_walker* w, const double* log_g, double factor, int continue_schedule) {
    for (uint64_t b = w->wb; b < w->we; ++b) w->log_g[b] = log_g[b];
    w->factor = factor;
    w->stage = factor <= w->p.final_factor ? WLG_STAGE_FROZEN : WLG_STAGE_WANG_LANDAU;
    w->time_offset = continue_schedule ? ORC_CONTINUE_SCHEDULE : 0;
}

orc_result* orc_run_rewl(const orc_couplings* c, const wlg_run_config* cfg, char* err, size_t len) {
    return orc_run_rewl_warm(c, cfg, NULL, 0.0, 0, err, len);
}

orc_result* orc_run_rewl_warm(const orc_couplings* c, const wlg_run_config* cfg, const double* warm_log_g,
                              double warm_factor, int continue_schedule, char* err, size_t len) {
    if (validate_config(cfg, 0, err, len)) return NULL;
    if (check_precision(cfg, err, len)) return NULL;
    if (cfg->coupling_precision == WLG_PRECISION_BF16 && c->csr) {
        set_err(err, len, "BF16 couplings are available for the dense backend only");
        return NULL;
    }
    uint64_t bins = 0;
    orc_grid_bins(cfg->emin, cfg->emax, cfg->bin_width, &bins);
    const uint64_t nw = cfg->windows, wpw = cfg->walkers_per_window, total = nw * wpw, n = c->n;
    uint64_t* windows = malloc(2 * nw * sizeof(uint64_t));
    if (cfg->explicit_windows) memcpy(windows, cfg->explicit_windows, 2 * nw * sizeof(uint64_t));
    else if (orc_partition_windows(bins, nw, cfg->overlap, windows)) {
        free(windows);
        set_err(err, len, "Invalid energy-window partition");
        return NULL;
    }
    orc_walker** ws = calloc(total, sizeof(orc_walker*));
    for (uint64_t w = 0; w < nw; ++w)
        for (uint64_t k = 0; k < wpw; ++k) {
            const uint64_t id = w * wpw + k;
            const int8_t* init = NULL;
            if (cfg->initial_spins && (!cfg->initial_spins_present || cfg->initial_spins_present[id]))
                init = cfg->initial_spins + id * n;
            char inner[2048] = {0};
            ws[id] = orc_walker_create(c, id, cfg->emin, cfg->emax, cfg->bin_width, windows[2 * w], windows[2 * w + 1],
                                       &cfg->wl, cfg->seed, init, inner, sizeof inner);
            if (!ws[id]) {
                set_err(err, len, "Walker initialization failed: window %llu, local walker %llu: %s",
                        (unsigned long long)w, (unsigned long long)k, inner);
                for (uint64_t q = 0; q < total; ++q) orc_walker_destroy(ws[q]);
                free(ws); free(windows);
                return NULL;
            }
        }
    if (warm_log_g)
        for (uint64_t q = 0; q < total; ++q) orc_walker_warm_start(ws[q], warm_log_g, warm_factor, continue_schedule);
    /* FP32 couplings: the constructors above used FP64; the updates from here on use FP32 */
    const int saved_update_fp32 = c->update_fp32, saved_update_bf16 = c->update_bf16;
    if (cfg->coupling_precision == WLG_PRECISION_FP32) ((orc_couplings*)c)->update_fp32 = 1;
    if (cfg->coupling_precision == WLG_PRECISION_BF16) orc_couplings_set_update_bf16((orc_couplings*)c, 1);
    const int checkpointing = cfg->checkpoint_path && cfg->checkpoint_path[0] && nw == 1 && wpw == 1;
    if (checkpointing) {
        int8_t* sp = malloc(n); double* fl = malloc(n * 8); double* lg = malloc(bins * 8);
        uint64_t* hs = malloc(bins * 8); uint8_t* ac = malloc(bins);
        wlg_snapshot snap;
        memset(&snap, 0, sizeof snap);
        char inner[512];
        if (load_checkpoint_into(cfg->checkpoint_path, ws[0], &snap, sp, fl, lg, hs, ac) == 0)
            orc_walker_restore(ws[0], &snap, inner, sizeof inner);
        free(sp); free(fl); free(lg); free(hs); free(ac);
    }
    orc_result* r = calloc(1, sizeof *r);
    uint64_t epoch = 0, last_checkpoint = 0;
    uint64_t* last_check = calloc(total, sizeof(uint64_t));
    const int unlimited = cfg->max_attempts == 0;
    const uint64_t ex = cfg->exchange_interval_attempts;
    const uint64_t recompute_epochs =
        cfg->coupling_precision != WLG_PRECISION_FP64 && cfg->recompute_interval_attempts != 0
            ? (cfg->recompute_interval_attempts + ex - 1) / ex
            : 0;
    int done = 0, status = 0;
    while (!done && !status) {
        int limit_reached = !unlimited;
        for (uint64_t w = 0; w < nw && !status; ++w) {
            for (uint64_t k = 0; k < wpw && !status; ++k) {
                orc_walker* x = ws[w * wpw + k];
                uint64_t batch = cfg->exchange_interval_attempts;
                if (!unlimited) {
                    const uint64_t remaining = x->attempted < cfg->max_attempts ? cfg->max_attempts - x->attempted : 0;
                    if (remaining < batch) batch = remaining;
                }
                status = orc_walker_run(x, batch, err, len);
            }
            if (!unlimited)
                for (uint64_t k = 0; k < wpw; ++k)
                    if (ws[w * wpw + k]->attempted < cfg->max_attempts) limit_reached = 0;
            const uint64_t ci = cfg->wl.check_interval_attempts > 1 ? cfg->wl.check_interval_attempts : 1;
            for (uint64_t k = 0; k < wpw && !status; ++k) {
                orc_walker* x = ws[w * wpw + k];
                if (x->stage != WLG_STAGE_WANG_LANDAU) continue;
                const uint64_t att = x->attempted;
                const int at_limit = !unlimited && att >= cfg->max_attempts;
                if (att - last_check[w * wpw + k] < ci && !at_limit) continue;
                last_check[w * wpw + k] = att;
                if (w_ready(x)) status = orc_walker_begin_next_iteration(x, err, len);
            }
        }
        if (status) break;
        const uint64_t parity = epoch % 2;
        for (uint64_t b = parity; b + 1 < nw && !status; b += 2) {
            for (uint64_t p = 0; p < wpw; ++p) {
                ++r->totals.exchange_attempted;
                int swapped = 0;
                status = local_exchange(ws[b * wpw + p], ws[(b + 1) * wpw + (p + epoch) % wpw], cfg->seed, epoch, b,
                                        &swapped, err, len);
                if (status) break;
                if (swapped) ++r->totals.exchange_accepted;
            }
        }
        ++epoch;
        int all_frozen_now = 1;
        for (uint64_t q = 0; q < total; ++q) all_frozen_now &= ws[q]->stage == WLG_STAGE_FROZEN;
        if (recompute_epochs && !(all_frozen_now || limit_reached) && epoch % recompute_epochs == 0)
            recompute_fp64(ws, total, c);
        if (checkpointing && ws[0]->attempted - last_checkpoint >= cfg->checkpoint_interval_attempts) {
            save_checkpoint(cfg->checkpoint_path, ws[0]);
            last_checkpoint = ws[0]->attempted;
        }
        int all_frozen = 1;
        for (uint64_t q = 0; q < total; ++q) all_frozen &= ws[q]->stage == WLG_STAGE_FROZEN;
        done = all_frozen || limit_reached;
    }
    free(last_check);
    ((orc_couplings*)c)->update_fp32 = saved_update_fp32;
    ((orc_couplings*)c)->update_bf16 = saved_update_bf16;
    if (status) {
        for (uint64_t q = 0; q < total; ++q) orc_walker_destroy(ws[q]);
        free(ws); free(windows); orc_result_destroy(r);
        return NULL;
    }
    r->totals.epochs = epoch;
    r->windows = nw; r->bins = bins; r->n = n;
    r->collect = cfg->wl.collect_window_statistics != 0;
    r->log_g = malloc(nw * bins * 8); r->histogram = malloc(nw * bins * 8);
    r->sem = malloc(nw * bins * 8); r->valid = malloc(nw * bins);
    r->stats = calloc(total, sizeof(wlg_walker_statistics));
    r->stat_count = total;
    r->round_trips = calloc(nw, 8);
    r->walker_counts = calloc(nw, 8);
    if (r->collect) {
        r->sq = calloc(nw * bins, 8); r->samples = calloc(nw * bins, 8);
        r->rep_energy = malloc(total * ORC_REPRESENTATIVES * 8);
        r->rep_spins = malloc(total * ORC_REPRESENTATIVES * n);
    }
    int converged = 1;
    for (uint64_t w = 0; w < nw && !status; ++w) {
        for (uint64_t k = 0; k < wpw; ++k) {
            orc_walker* x = ws[w * wpw + k];
            r->totals.attempted += x->attempted;
            r->totals.accepted += x->accepted;
            r->totals.forced_accepted += x->forced;
            converged &= x->stage == WLG_STAGE_FROZEN;
            wlg_histogram_statistics h;
            orc_walker_histogram_statistics(x, &h);
            wlg_walker_statistics* s = &r->stats[w * wpw + k];
            s->walker_id = x->id; s->window_id = w; s->mpi_rank = 0;
            s->attempted = x->attempted; s->accepted = x->accepted; s->forced_accepted = x->forced;
            s->attempts_since_last_accepted = x->attempted - x->last_acc;
            s->energy = x->energy; s->factor = x->factor; s->active_bins = h.active_bins;
            s->minimum_histogram = h.minimum; s->mean_histogram = h.mean; s->min_over_mean = h.min_over_mean;
            s->round_trips = x->round_trips;
            if (r->collect)
                for (int q = 0; q < ORC_REPRESENTATIVES; ++q)
                    if (x->rep_present[q]) {
                        r->rep_energy[r->rep_count] = x->rep_energy[q];
                        memcpy(r->rep_spins + r->rep_count * n, x->rep_spins + (uint64_t)q * n, n);
                        ++r->rep_count;
                    }
        }
        status = summarize(ws + w * wpw, wpw, windows[2 * w], windows[2 * w + 1], bins, r->collect,
                           r->log_g + w * bins, r->histogram + w * bins, r->sem + w * bins, r->valid + w * bins,
                           err, len);
        r->walker_counts[w] = wpw;
        if (r->collect)
            for (uint64_t k = 0; k < wpw; ++k) {
                orc_walker* x = ws[w * wpw + k];
                for (uint64_t i = windows[2 * w]; i < windows[2 * w + 1]; ++i) {
                    r->sq[w * bins + i] += x->sqdisp[i];
                    r->samples[w * bins + i] += x->dsamples[i];
                }
                r->round_trips[w] += x->round_trips;
            }
    }
    r->totals.converged = converged;
    for (uint64_t q = 0; q < total; ++q) orc_walker_destroy(ws[q]);
    free(ws); free(windows);
    if (status) { orc_result_destroy(r); return NULL; }
    return r;
}

void orc_result_totals(const orc_result* r, wlg_run_totals* out) { *out = r->totals; }

int orc_result_fragment(const orc_result* r, uint64_t w, double* log_g, uint64_t* hist, double* sem, uint8_t* valid) {
    if (w >= r->windows) return WLG_ERR_OUT_OF_RANGE;
    memcpy(log_g, r->log_g + w * r->bins, r->bins * 8);
    memcpy(hist, r->histogram + w * r->bins, r->bins * 8);
    memcpy(sem, r->sem + w * r->bins, r->bins * 8);
    memcpy(valid, r->valid + w * r->bins, r->bins);
    return 0;
}

uint64_t orc_result_walker_statistics(const orc_result* r, wlg_walker_statistics* out, uint64_t capacity) {
    const uint64_t count = capacity < r->stat_count ? capacity : r->stat_count;
    memcpy(out, r->stats, count * sizeof *out);
    return r->stat_count;
}

int orc_result_sampling(const orc_result* r, uint64_t w, double* sq, uint64_t* samples, uint64_t* round_trips,
                        uint64_t* walkers) {
    if (!r->collect || w >= r->windows) return WLG_ERR_OUT_OF_RANGE;
    memcpy(sq, r->sq + w * r->bins, r->bins * 8);
    memcpy(samples, r->samples + w * r->bins, r->bins * 8);
    *round_trips = r->round_trips[w];
    *walkers = r->walker_counts[w];
    return 0;
}

uint64_t orc_result_representatives(const orc_result* r, double* energies, int8_t* spins, uint64_t capacity) {
    const uint64_t count = capacity < r->rep_count ? capacity : r->rep_count;
    if (count) {
        memcpy(energies, r->rep_energy, count * 8);
        memcpy(spins, r->rep_spins, count * r->n);
    }
    return r->rep_count;
}

/* exact_enumeration (src/analysis.cpp:162-181) */
int orc_exact_enumeration(const orc_couplings* c, double emin, double emax, double width, uint64_t* counts) {
    const uint64_t n = c->n;
    if (n > 26 || n >= 63) return WLG_ERR_INVALID_ARGUMENT;
    uint64_t bins = 0;
    if (orc_grid_bins(emin, emax, width, &bins)) return WLG_ERR_INVALID_ARGUMENT;
    memset(counts, 0, bins * 8);
    int8_t* spins = malloc(n);
    const uint64_t states = (uint64_t)1 << n;
    for (uint64_t state = 0; state < states; ++state) {
        for (uint64_t i = 0; i < n; ++i) spins[i] = (state & ((uint64_t)1 << i)) ? 1 : -1;
        const int64_t b = orc_grid_index(emin, emax, width, orc_total_energy(c, spins));
        if (b >= 0) ++counts[b];
    }
    free(spins);
    return 0;
}
