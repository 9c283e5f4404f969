/* Oracle: hand-written CPU restatement of ThunderEngine's CM1 large-step dynamics
 * kernels (data/kernels/*.wgsl of the reference), TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
 * library.  The product (include/thunderstep.h) never links it.
 *
 * Calling convention = the reference player's (web/replay.js:258-288): one word memory
 * M and a 64-word argument slot ARG per dispatch: ARG[0..2] grid in threads,
 * ARG[3] = 0, ARG[4+n] = word offset of binding n.  Every kernel is exported as
 *     void teor_<kernel name>(uint32_t *M, const uint32_t *ARG);
 * Arithmetic is IEEE binary32; the reference's numbers assume subnormals are flushed
 * (FTZ/DAZ), so callers enable that with te_set_ftz(1) first.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint32_t te_fnv1a(const uint32_t *w, size_t n);
void te_set_ftz(int on);
float te_div_cr(float a, float b);
float te_sqrt_cr(float x);
float te_weno5(float s1, float s2, float s3, float s4, float s5, float weps);
float te_rr_pow_cr(float x, float p);

#define TE_ORACLE_KERNEL(name) void teor_##name(uint32_t *M, const uint32_t *ARG);
float te_pow_f64(float x, float y);
float te_exp_f64(float x);
float te_log_f64(float x);
float te_log2_f64(float x);
float te_atan2_f64(float y, float x);

#define TE_ORACLE_KERNELS(X) \
  X(adv_flux_x) X(adv_flux_y) X(adv_flux_z) \
  X(adv_flux_x_stag) X(adv_flux_y_stag) X(adv_flux_z_stag) \
  X(adv_flux_x_weno) X(adv_flux_y_weno) X(adv_flux_z_weno) \
  X(adv_flux_x_weno_uv) X(adv_flux_y_weno_uv) X(adv_flux_z_weno_uv) \
  X(adv_flux_x_weno_w) X(adv_flux_y_weno_w) X(adv_flux_z_weno_w) \
  X(adv_assemble) X(rk_update) X(pdef_dum) X(pdef_apply) \
  X(build_sadv) X(massflux_from_state) X(div_massflux) X(velocity_to_massflux) \
  X(stage_state_reset) X(stage_tendency_reset) X(buoyancy_apply) X(apply_thterm) \
  X(acoustic_prepare) X(acoustic_begin) X(acoustic_uv) X(acoustic_fpk) \
  X(acoustic_w_solve) X(acoustic_pp) X(acoustic_accumulate) \
  X(bc_periodic_x) X(bc_periodic_y) \
  X(update_diagnostics) X(stability_max) X(update_diagnostics_moist) X(pressure_tendency) X(divergence3d) \
  X(update_rho_prs) X(diabatic_unapply) X(diabatic_rates) X(ppx_finish) \
  X(bc_open_x) X(bc_open_y) X(radbc_ew) X(radbc_ns) X(openbc_uv_tendency) \
  X(turb_zero) X(turb_add_tendency) X(turb_scalar_flux_h) X(turb_openbc_flux) \
  X(turb_openbc_stress_x) X(turb_openbc_stress_y) X(tke_advance) X(tke_sources) X(tke_flux_h) \
  X(mp_pdefq) X(turb_scalar_vert_implicit) \
  X(rayleigh_damping) X(turb_rho_faces) X(turb_def_centers) X(turb_def_faces) X(turb_def_assemble) \
  X(turb_gettau) X(turb_km_kh) X(tke_epst) \
  X(turb_nm) X(turb_sfcstress) X(turb_dissipative_heating) \
  X(turb_u_tendency) X(turb_v_tendency) X(turb_w_tendency) X(tke_transport) \
  X(mass_row_sums) X(mass_level_sums) X(mass_reference_init) X(mass_correction_apply) \
  X(morr_prep) X(morr_post)
TE_ORACLE_KERNELS(TE_ORACLE_KERNEL)

#ifdef __cplusplus
}
#endif
