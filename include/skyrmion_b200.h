/* skyrmion_b200 — C ABI of the B200-native (sm_100a) skyrmion_solver lattice engine.
 *
 * Every entry point takes plain pointers and sizes; device buffers are raw
 * CUDA device pointers, "host" arguments are host pointers, `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Calls are asynchronous on
 * `stream` unless an output is a host pointer, in which case the call
 * synchronises that stream before returning.
 *
 * Parameter ABI: `p_i` (int32, n_pi entries) and `p_f` (float64, n_pf entries)
 * are the reference's packed parameter arrays (skyrmion_solver
 * core/params.py:227-267 plus the theory's pack_device_params):
 *   p_i = [xlen, ylen, zlen, halo, ncoord, nfields, dim_grid, dim_fields,
 *          killkinen, newtonflow, unit_length, <theory ints...>]
 *   p_f = [xsize, ysize, zsize, lsx, lsy, lsz, grid_volume, time_step,
 *          <theory couplings...>]
 * Field buffers use the reference layout: FP64, index a*N + x*Y*Z + y*Z + z.
 *
 * Return value: a sky_status (0 = success).
 */
#ifndef SKYRMION_B200_H
#define SKYRMION_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SKY_OK = 0,
    SKY_ERR_INVALID = 1,   /* bad argument: sizes, parameter arrays, theory id */
    SKY_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    SKY_ERR_NONFINITE = 3, /* reserved: non-finite energies are returned as values, as the
                              reference returns them (its step reports NaN, it does not raise) */
    SKY_ERR_TIMEOUT = 4,   /* a stage kernel gave up a bounded wait for a TMA plane copy (the
                              engine's statistics calls report it; the step is not valid) */
    SKY_ERR_NOMEM = 5      /* caller-provided scratch too small / allocation failed */
} sky_status;

typedef enum {
    SKY_THEORY_NUCLEAR = 0,       /* th/nuclear_skyrme        C = 4  */
    SKY_THEORY_OMEGA = 1,         /* th/omega_skyrme          C = 5  */
    SKY_THEORY_COULOMB = 2,       /* th/coulomb_skyrme        C = 5  */
    SKY_THEORY_RHO = 3,           /* th/rho_skyrme            C = 13 */
    SKY_THEORY_BERGER = 4,        /* th/berger_skyrme         C = 4  */
    SKY_THEORY_LIGHTLY_BOUND = 5  /* th/lightly_bound_skyrme  C = 4  */
} sky_theory;

/* Library version string and the last CUDA error text seen by this thread. */
const char* sky_version(void);
const char* sky_last_error(void);

/* Library-wide tuning options.  Key 0: kernel family of the reference-layout
 * gradient (sky_gradient_step / sky_arrested_newton_step) for theories with at
 * most five components: 1 = marching x-plane kernels (default), 0 = 3-D tile
 * kernels.  Key 1: x-chunk of those marching launches (0 = automatic).  Key 2:
 * staging of the resident engine's stage kernels, 1 = tensor-memory-accelerator
 * box copies (default; lattices whose Z gives 16-byte row pitches), 0 = per-thread
 * cp.async copies; it applies to instances admitted afterwards
 * (sky_engine_set_staging changes one instance).
 * Key 3: 1 = the FP32 stages of theories whose gradient needs no mixed second
 * derivatives (omega) compute two adjacent z-sites per thread with packed FP32x2
 * arithmetic; 0 = one site per thread (default).  Applies at admission.
 * Key 4: 1 = the engine's stage launches use programmatic dependent launch, so a
 * launch is scheduled while the previous one's last blocks finish (each waits for
 * the previous launch before reading its results), 0 = plain stream order (default;
 * inside the step graphs the two measure the same).
 * It applies to the next step call (captured graphs are rebuilt).
 * Process-wide; not synchronised with launches in flight on other threads. */
int sky_set_option(int key, int value);
int sky_get_option(int key);

/* Number of field components the theory's kernels are built for. */
int sky_theory_components(int theory);

/* Doubles of scratch that sky_sum / sky_max / sky_total_* need for n values. */
int64_t sky_reduce_scratch_size(int64_t n);

/* ------------------------------------------------------------------------ *
 * Reference-layout FP64 kernels (drop-ins for the reference's launches).
 * ------------------------------------------------------------------------ */

/* Replaces the theory's do_gradient_step_kernel
 * (core/integrator.py:37-46 + th/<theory>/kernels.py: do_gradient_step_point):
 * EG = projected energy gradient of `field`, l_out = -time_step * EG.
 * The reference's d1fd1x / d2fd2x scratch buffers are not needed. */
int sky_gradient_step(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                      double* l_out, const double* field, double* energy_gradient, void* stream);

/* Replaces do_rk4_step_kernel (core/integrator.py:50-92):
 * k_out = dt (velocity + factor l_in); temp = field + factor k_prev. */
int sky_rk4_stage(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* k_out,
                  const double* velocity, const double* l_in, double* temp, const double* field,
                  const double* k_prev, double factor, void* stream);

/* Replaces the theory's do_rk4_kernel (core/integrator.py:163-175 with the
 * theory's norm / projection).  theory < 0 selects do_rk4_kernel_no_constraint
 * (core/integrator.py:94-141). */
int sky_rk4_finalize(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                     double* velocity, double* field, const double* k1, const double* k2, const double* k3,
                     const double* k4, const double* l1, const double* l2, const double* l3, const double* l4,
                     void* stream);

/* Replaces compute_energy_kernel (e.g. th/nuclear_skyrme/kernels.py:350-382): en = e * h^3. */
int sky_energy_density(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                       double* en, const double* field, void* stream);

/* Replaces compute_skyrmion_number_kernel (e.g. th/nuclear_skyrme/kernels.py:450-482). */
int sky_baryon_density(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                       double* en, const double* field, void* stream);

/* Replaces compute_potential_kernel (th/omega_skyrme/kernels.py:413-441,
 * th/coulomb_skyrme/kernels.py:417-445): en = field component p_i[11]. */
int sky_potential_density(const int32_t* p_i, int32_t n_pi, double* en, const double* field, void* stream);

/* Replaces compute_rho_meson_kernel (th/rho_skyrme/kernels.py:385-412): en += sum_{a>=4} field_a^2. */
int sky_rho_meson_density(const int32_t* p_i, int32_t n_pi, double* en, const double* field, void* stream);

/* Replaces set_field_zero_kernel (core/utils.py:148-174). */
int sky_set_field_zero(const int32_t* p_i, int32_t n_pi, double* field, void* stream);

/* Replaces create_grid_kernel (e.g. th/nuclear_skyrme/kernels.py:27-56): grid_i = h_i * index. */
int sky_create_grid(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* grid,
                    void* stream);

/* Baryon moments for the reference's compute_center_of_mass / compute_rms_radius
 * (th/nuclear_skyrme/observables.py:182-270 with compute_center_of_mass_kernel
 * and compute_rms_radius_kernel, th/nuclear_skyrme/kernels.py:678-758), in one
 * fused pass: with b the per-site baryon density (h^3 included) and r the grid
 * point (h_x i, h_y j, h_z k), out9_host = [sum b, sum b r (3), sum |b|,
 * sum |b| r (3), sum |b| |r|^2] (compensated FP64, deterministic).  Then
 * COM = sum b r / sum b and RMS^2 = sum |b| |r - COM|^2 / sum b.  scratch: a
 * device buffer of sky_reduce_scratch_size() doubles.  Synchronous. */
int sky_baryon_moments(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                       const double* field, double* scratch, int64_t n_scratch, double* out9_host, void* stream);

/* The nuclear model's inertia and shape diagnostics (compute_U_tensor,
 * compute_V_tensor, compute_W_tensor, compute_quadrupole_tensor and the
 * D-term integral of compute_D_term; th/nuclear_skyrme/observables.py:273-487
 * with kernels.py:484-1033) in one fused FP64 pass, about the centre of mass
 * com_host (host, 3 doubles; e.g. from sky_baryon_moments).  out28_host =
 * [U00 U01 U02 U11 U12 U22, V (the same six), W00..W22 (nine, row-major),
 * Q (six, as U), D integral], compensated and deterministic; the D-term is
 * -(2/5) E times the last entry.  scratch: sky_reduce_scratch_size() doubles.
 * Synchronous. */
int sky_nuclear_diagnostics(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                            const double* field, const double* com_host, double* scratch, int64_t n_scratch,
                            double* out28_host, void* stream);

/* Initial field on the device (replaces the reference's initial-configuration
 * kernels, th/nuclear_skyrme/initial_config.py:583-627, 664-698, 941-953,
 * 1082-1126): the normalised quaternion product, in order, of nsol <= 48
 * solitons with profile f(r) = pi exp(-r / scale).  Soliton k has baryon
 * number baryon[k] (1: hedgehog; 2 or 4: the rational maps z^2 and the cubic
 * map), centre centers[3k..3k+2] and isorotation quats[4k..4k+3] (unit
 * quaternion; quats may be NULL).  nsol = 0 gives the vacuum.  Components
 * 4..C-1 are zeroed, and the outer vacuum_shell sites of every face are set to
 * the vacuum.  field: device buffer of C*N doubles. */
int sky_init_field(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, int32_t nsol,
                   const int32_t* baryon, const double* centers, const double* quats, double scale,
                   int32_t vacuum_shell, double* field, void* stream);

/* Replaces the reference's initial configurations (th/<theory>/initial_config.py:
 * create_ground_state_kernel, create_initial_configuration_kernel, and the
 * smorgasbord's create_rational_map_skyrmion_kernel + product_ansatz_kernel).
 * Field components 0..3 become the product, in list order, of n_lumps lumps,
 * each normalised and each product normalised; components 4.. become 0.  With
 * from_vacuum != 0 the product starts from (1, 0, 0, 0) and composes every lump
 * (the smorgasbord); otherwise it starts from the first lump itself (the single
 * ansatz).  n_lumps = 0 gives the vacuum.  Each lump is 16 doubles:
 *   [0] kind: 0 Gaussian hedgehog pi exp(-(r / r0)^2) (hedgehog_field),
 *             1 rational map with the fitted profile (profilefun, rational_map_value)
 *   [1] baryon number (the map's R_B and profile, rounded, >= 1)
 *   [2..4] centre in grid coordinates (x_i = h i)
 *   [5..7] Euler angles z, y, z applied to the position (maps only)
 *   [8..10] Euler angles applied to the target direction (hedgehog: [10] about z)
 *   [11] profile length r0 > 0 (maps: the profile is evaluated at r / r0)
 *   [12] profile mass mixing m0 (maps; below 1 blends the massless fit)
 *   [13..15] unused (0). */
int sky_init_lumps(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, int32_t n_lumps,
                   const double* lumps, int32_t from_vacuum, double* field, void* stream);

/* Replace the viewer's volume builder (build_rgba_volume_kernel with the
 * extrema of _reduce_density_extrema, th/nuclear_skyrme/render_gl.py:157-222,
 * 447-500): volume[((z * Y + y) * X + x) * 4 + c] (FP32) holds the density
 * normalised to its [min, max] (c = 0) and the unit pion vector (c = 1..3;
 * (0, 0, 1) where |pi|^2 <= 1e-20).  `density` holds N FP64 values, `field`
 * the reference-layout field (C >= 4).  `scratch` holds at least
 * sky_volume_scratch_size() doubles; once the stream reaches the end of the
 * call, scratch[0] and scratch[1] hold the density minimum and maximum.  If
 * minmax_host is not NULL, they are also copied there and the stream is
 * synchronised; otherwise the call is asynchronous. */
int64_t sky_volume_scratch_size(void);
int sky_build_rgba_volume(const int32_t* p_i, int32_t n_pi, const double* density, const double* field,
                          double* scratch, int64_t n_scratch, float* volume, double* minmax_host, void* stream);

/* Replaces the viewer's ray-march fragment shader
 * (visualization/gl_backend.py:519-710) without a graphics API: image[(row *
 * width + col) * 4 + c] (FP32 RGBA, row 0 at the top) from the volume above
 * (xlen * ylen * zlen texels, trilinear, clamp to edge).  params (host,
 * n_params >= 23 floats): the three inverse-view rows (12), box scale (3), zoom,
 * brightness, levelset, density min, density max, transfer scale, opacity scale,
 * tstep.
 * color_mode 0 uses the viewer's nine-entry transfer table; any other value
 * the pion vector's HSL colour.  Rays that miss the box give (1, 1, 1, 1). */
int sky_render_volume(const float* volume, int32_t xlen, int32_t ylen, int32_t zlen, const float* params,
                      int32_t n_params, int32_t max_steps, int32_t color_mode, int32_t width, int32_t height,
                      float* image, void* stream);

/* Replace compute_sum / compute_max (core/utils.py:201-279, 321-373):
 * deterministic FP64 reductions (compensated sum; signed max).  `scratch` is a
 * device buffer of sky_reduce_scratch_size(n) doubles; the result is written to
 * *out_host (host pointer; the stream is synchronised) and, if out_dev is not
 * NULL, also to out_dev[0] on the device. */
int sky_sum(const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host,
            double* out_dev, void* stream);
int sky_max(const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host,
            double* out_dev, void* stream);

/* Replaces compute_min (core/utils.py:282-319, 375-400): the minimum of n values,
 * exact (the negated maximum of the negated values).  Same buffers as sky_max. */
int sky_min(const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host,
            double* out_dev, void* stream);

/* Replaces arresting_criteria and arresting_criteria_kernel
 * (core/integrator.py:178-282): per site the power sum_a V_a EG_a (written to en
 * if it is not NULL) and its compensated sum over the lattice, into *out_host
 * (synchronous) when out_host is not NULL.  scratch: sky_reduce_scratch_size()
 * doubles. */
int sky_arresting_criteria(const int32_t* p_i, int32_t n_pi, const double* velocity, const double* energy_gradient,
                           double* en, double* scratch, int64_t n_scratch, double* out_host, void* stream);

/* Replace the host compute_energy / compute_skyrmion_number
 * (th/nuclear_skyrme/observables.py:408-474): the per-site density and its
 * compensated FP64 sum fused into one launch (no per-site buffer round trip). */
int sky_total_energy(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                     const double* field, double* scratch, int64_t n_scratch, double* out_host, void* stream);
int sky_total_baryon(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                     const double* field, double* scratch, int64_t n_scratch, double* out_host, void* stream);

/* Replaces do_arrested_newton_flow (core/integrator.py:284-410): one RK4 step of
 * the arrested Newton flow with the reference's buffers and semantics (k1..k4,
 * l1..l4, temp and energy_gradient hold the same content afterwards; velocity is
 * zeroed when killkinen and the new energy exceeds prev_energy).  Writes the new
 * energy and err (signed max of the stage-4 gradient) to host pointers. */
int sky_arrested_newton_step(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                             double* velocity, double* field, double* energy_gradient, double* k1, double* k2,
                             double* k3, double* k4, double* l1, double* l2, double* l3, double* l4, double* temp,
                             double* scratch, int64_t n_scratch, double prev_energy, double* new_energy_host,
                             double* err_host, void* stream);

/* No counterpart in the reference.  The same step as sky_arrested_newton_step
 * for callers that cannot allocate device memory: a plugin handed only the
 * field and velocity of a host application whose allocator owns the device
 * memory, or an interactive loop that must not call cudaMalloc / cudaFree
 * (they synchronise the device) between frames.  The eight RK4 slopes, the
 * stage field and the reduction scratch live in a 16 MiB static device array
 * that every GPU loading the library holds until exit, so the lattice is
 * limited to C*N <= 232488 values (e.g. 35^3 sites at C = 5); larger lattices
 * are rejected with SKY_ERR_INVALID before anything is launched.  The array's
 * device address is looked up on the first call on each device, and again on
 * the first call after the device's context was re-created (cudaDeviceReset
 * reloads the library's module), so make that first call before any stream
 * capture.  All calls share the array: calls
 * that overlap on the GPU (other streams, other threads) race.  The slopes are
 * not returned; velocity, field and energy_gradient are updated as by
 * sky_arrested_newton_step, and the new energy and err go to host pointers. */
int sky_arrested_newton_step_noalloc(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                                     double* velocity, double* field, double* energy_gradient, double prev_energy,
                                     double* new_energy_host, double* err_host, void* stream);

/* ------------------------------------------------------------------------ *
 * Resident batched engine.  No reference counterpart as a single call: it
 * runs the arrested-Newton step of core/integrator.py:284-410 (driven in the
 * reference by Simulation.step, core/simulation.py:287-308) for many
 * instances at once, entirely on the device, with fused RK4 stages, FP64
 * compensated energy / baryon reductions, a device-side arrest decision and
 * CUDA-graph replay.  The engine owns its device memory.
 * ------------------------------------------------------------------------ */

/* Create / destroy an engine bound to CUDA device `device`. */
int sky_engine_create(int device, void** engine_out);
int sky_engine_destroy(void* engine);

/* Admit one instance.  precision: 0 = FP32 state and stage arithmetic,
 * 1 = FP64, 2 = FP32 stage arithmetic with a compensated field (stored as an
 * unevaluated FP32 sum hi + lo and updated in FP64 at the end of each step, so
 * that near convergence updates far below one FP32 ulp still accumulate; the
 * stencils read hi only), 3 = as 2 with a defect-corrected gradient: every 16
 * steps an FP64 gradient of hi + lo is evaluated and the difference to the FP32
 * gradient of the same field is added to every stage's FP32 gradient until the
 * next refresh, so the flow's fixed point is the FP64 one while the stencils stay
 * FP32 (every theory; rho's thirteen-component FP64 refresh walks 4-row sub-tiles).
 * field / velocity are FP64 in the reference layout (host pointers,
 * or device pointers when on_device != 0); velocity may be NULL (zero).  The
 * energy of the admitted field is evaluated immediately (stats record 0). */
int sky_engine_add(void* engine, int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                   int precision, const double* field, const double* velocity, int on_device, int* id_out);

/* Retire an instance and free its memory. */
int sky_engine_remove(void* engine, int id);

/* Change an instance's precision (0..3 as for sky_engine_add) in place,
 * e.g. to FP64 for the polishing phase; the field, velocity, step count and
 * pending arrest decision carry over. */
int sky_engine_set_precision(void* engine, int id, int precision);

/* Re-tile an instance: x-chunk `xc` planes per block of the marching kernels
 * (0 = automatic choice from the grid and the SM count).  The state and the
 * pending arrest decision carry over. */
int sky_engine_retile(void* engine, int id, int xc);
/* Staging of an instance's planes in the marching stage kernels: tma = 1 copies
 * each haloed plane with one tensor-memory-accelerator box copy per source (Z *
 * element size a multiple of 16 bytes; not FP64 rho), 0 with per-thread cp.async
 * copies; pair = 1 runs two z-sites per thread with packed FP32x2 arithmetic (TMA,
 * FP32 omega only).  Admission takes both from library options 2 and 3; a group of
 * instances of one theory and precision stages by TMA (z-pairs) only when every
 * member does.  The state and the pending arrest decision carry over; the
 * stagings are bitwise identical, z-pairs agree to FP32 rounding. */
int sky_engine_set_staging(void* engine, int id, int tma, int pair);
int sky_engine_get_staging(void* engine, int id, int* tma, int* pair);
/* Steps between refreshes of a defect-corrected instance's FP64 correction
 * (precision 3; default 16, period >= 1).  A shorter period follows a field
 * that moves (a drifting soliton) at the cost of more FP64 gradient passes. */
int sky_engine_set_defect_period(void* engine, int id, int period);
/* Current x-chunk of an instance (-1 if unknown). */
int sky_engine_get_xc(void* engine, int id);

/* Energy audit of the RK4 dynamics (killkinen = 0) of an instance's current
 * state, in FP64 (synchronous).  out2 = [Phi, K]: Phi is the potential whose
 * (anti-)gradient the kernels integrate and K = (1/2) h^3 sum_c s_c |V_c|^2;
 * H = Phi + K is conserved up to the O(h^4) gap between the force and energy
 * stencils.  For the nuclear, rho, Berger and lightly-bound variants Phi is
 * the coded energy and s_c = 1; for omega, Phi = E_pion - E_omega -
 * c_omega omega B0, and for Coulomb, Phi = E_pion/2 - (kappa/2)|grad A0|^2 +
 * kappa A0 B0, both with s_4 = -1 (the auxiliary field is the time component
 * of a vector field).  No reference counterpart: the reference's dynamics
 * reports only the coded energy (core/simulation.py:287-308). */
int sky_engine_audit(void* engine, int id, double* out2);

/* Pause (0) or resume (1) an instance. */
int sky_engine_set_active(void* engine, int id, int active);

/* Advance every active instance by nsteps arrested-Newton steps (asynchronous). */
int sky_engine_step(void* engine, int nsteps);
int sky_engine_synchronize(void* engine);
void* sky_engine_stream(void* engine);

/* Statistics after `step` steps of instance id (step < 0: the latest):
 * out6 = [energy, baryon, err (signed max of the step's stage-4 gradient),
 *         max|gradient|, arrested (velocity zeroed for the next step), step]. */
int sky_engine_stats(void* engine, int id, int64_t step, double* out6);

/* As sky_engine_stats, with out8 = [energy, baryon, err, max|g|, arrested, step,
 * kinetic energy (1/2) h^3 sum |V|^2 of the velocity the step produced (before any
 * arrest; with killkinen = 0 this is the RK4 dynamics' kinetic energy),
 * precision (0..3)]. */
int sky_engine_stats_ex(void* engine, int id, int64_t step, double* out8);

/* Latest statistics of up to `cap` instances: ids_out[k] and out7[7k..7k+6] =
 * [energy, baryon, err, max|g|, arrested, step, precision]; returns the count
 * through *count_out. */
int sky_engine_stats_all(void* engine, int* ids_out, double* out7, int cap, int* count_out);

/* Copy an instance's field and velocity out as FP64 in the reference layout
 * (host pointers, or device pointers when on_device != 0); either may be NULL.
 * The velocity reads as zero when the last step arrested it, as in the reference. */
int sky_engine_read(void* engine, int id, double* field, double* velocity, int on_device);

/* Run nsteps steps without graph capture, timing each launch kind with CUDA
 * events on the engine stream; ms_out[6] = average milliseconds per step spent
 * in [stage 1 (with the defect refresh and the folded control), stage 2, stage 3,
 * stage 4 + update (with the folded advance), 0, 0]: the last two entries (the
 * separate control and advance launches) are kept for compatibility. */
int sky_engine_time_stages(void* engine, int nsteps, double* ms_out);

/* Kernel launches one step issues: 4 per non-empty (theory, precision) group
 * (stages 2, 3, 4 and 1; stage 4's last block per instance advances it and stage
 * 1's runs its control), 5 when the group holds a defect-corrected instance. */
int sky_engine_launches_per_step(void* engine);

int sky_engine_count(void* engine);
int64_t sky_engine_bytes(void* engine);

#ifdef __cplusplus
}
#endif

#endif /* SKYRMION_B200_H */
