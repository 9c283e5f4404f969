/* Binary64 CPU adjoint of the dynamics-core step (TEST INFRASTRUCTURE ONLY, like oracle.c).
 *
 * The adjoint operators of the library (thunderengine-web_b200/csrc/te_adjoint.cuh)
 * instantiated in binary64 over the binary64 twin's value memory D (one double per
 * memory word, oracle/oracle64.c), with the adjoint memory L of the same layout.  It is
 * the "FP64 CPU adjoint" the GPU's binary32 gradient is compared with; its correctness is
 * checked independently against binary64 central differences of the twin's forward step.
 *
 *   void teadj_run(const char *name, const uint32_t *M, double *D, double *L,
 *                  const uint32_t *ARG, uint64_t ptr_mask, int acoustic)
 * runs the adjoint of one dispatch: ARG is the player's slot (grid in threads, word
 * offsets of the bindings), ptr_mask bit n marks binding n as a field pointer (others are
 * setBytes structs read from M), `acoustic` marks binding 1 as AcousticParams.
 * Returns through the memory; unknown names set *teadj_error. */
#include <omp.h>

#include <cstdint>
#include <cstring>

#include "../thunderengine-web_b200/csrc/te_adjoint.cuh"

using namespace te;
using namespace te::adj;

namespace {

struct AccHost {
  static constexpr bool skip_zero = true;
  static inline void add(double *p, double v) {
#pragma omp atomic
    *p += v;
  }
  static inline void add(float *p, float v) {
#pragma omp atomic
    *p += v;
  }
};

inline float wordf(uint32_t w) {
  float x;
  std::memcpy(&x, &w, 4);
  return x;
}

template <void (*Fn)(const AdjArgs<double> &, int, int, int)>
void loop(const AdjArgs<double> &A) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int tz = 0; tz < A.gz; tz++)
    for (int ty = 0; ty < A.gy; ty++)
      for (int tx = 0; tx < A.gx; tx++) Fn(A, tx, ty, tz);
}

#define DIR(f, d) \
  [](const AdjArgs<double> &A, int x, int y, int z) { f<double, AccHost>(A, x, y, z, d); }

typedef void (*Runner)(const AdjArgs<double> &);

template <void (*Fn)(const AdjArgs<double> &, int, int, int)>
Runner runner() {
  return loop<Fn>;
}

void fx(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_lin_h<double, AccHost>(A, x, y, z, 0); }
void fy(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_lin_h<double, AccHost>(A, x, y, z, 1); }
void sx(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_stag_h<double, AccHost>(A, x, y, z, 0); }
void sy(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_stag_h<double, AccHost>(A, x, y, z, 1); }
void wx(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_weno_h<double, AccHost>(A, x, y, z, 0); }
void wy(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_weno_h<double, AccHost>(A, x, y, z, 1); }
void uvx(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_weno_uv_h<double, AccHost>(A, x, y, z, 0); }
void uvy(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_weno_uv_h<double, AccHost>(A, x, y, z, 1); }
void wwx(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_weno_w_h<double, AccHost>(A, x, y, z, 0); }
void wwy(const AdjArgs<double> &A, int x, int y, int z) { adj_flux_weno_w_h<double, AccHost>(A, x, y, z, 1); }
void hx(const AdjArgs<double> &A, int x, int y, int z) { adj_bc_periodic<double, AccHost>(A, x, y, z, 0); }
void hy(const AdjArgs<double> &A, int x, int y, int z) { adj_bc_periodic<double, AccHost>(A, x, y, z, 1); }

struct Entry {
  const char *name;
  Runner run;
};

const Entry kTable[] = {
    {"adv_flux_x", runner<fx>()},
    {"adv_flux_y", runner<fy>()},
    {"adv_flux_z", runner<adj_flux_lin_z<double, AccHost>>()},
    {"adv_flux_x_stag", runner<sx>()},
    {"adv_flux_y_stag", runner<sy>()},
    {"adv_flux_z_stag", runner<adj_flux_stag_z<double, AccHost>>()},
    {"adv_flux_x_weno", runner<wx>()},
    {"adv_flux_y_weno", runner<wy>()},
    {"adv_flux_z_weno", runner<adj_flux_weno_z<double, AccHost>>()},
    {"adv_flux_x_weno_uv", runner<uvx>()},
    {"adv_flux_y_weno_uv", runner<uvy>()},
    {"adv_flux_z_weno_uv", runner<adj_flux_weno_uv_z<double, AccHost>>()},
    {"adv_flux_x_weno_w", runner<wwx>()},
    {"adv_flux_y_weno_w", runner<wwy>()},
    {"adv_flux_z_weno_w", runner<adj_flux_weno_w_z<double, AccHost>>()},
    {"adv_assemble", runner<adj_assemble<double, AccHost>>()},
    {"rk_update", runner<adj_rk_update<double, AccHost>>()},
    {"apply_thterm", runner<adj_apply_thterm<double, AccHost>>()},
    {"buoyancy_apply", runner<adj_buoyancy_apply<double, AccHost>>()},
    {"update_diagnostics_moist", runner<adj_update_diagnostics_moist<double, AccHost>>()},
    {"stage_tendency_reset", runner<adj_stage_tendency_reset<double, AccHost>>()},
    {"massflux_from_state", runner<adj_massflux_from_state<double, AccHost>>()},
    {"div_massflux", runner<adj_div_massflux<double, AccHost>>()},
    {"divergence3d", runner<adj_divergence3d<double, AccHost>>()},
    {"velocity_to_massflux", runner<adj_velocity_to_massflux<double, AccHost>>()},
    {"build_sadv", runner<adj_build_sadv<double, AccHost>>()},
    {"stage_state_reset", runner<adj_stage_state_reset<double, AccHost>>()},
    {"acoustic_begin", runner<adj_acoustic_begin<double, AccHost>>()},
    {"acoustic_prepare", runner<adj_acoustic_prepare<double, AccHost>>()},
    {"acoustic_uv", runner<adj_acoustic_uv<double, AccHost>>()},
    {"acoustic_fpk", runner<adj_acoustic_fpk<double, AccHost>>()},
    {"acoustic_pp", runner<adj_acoustic_pp<double, AccHost>>()},
    {"acoustic_accumulate", runner<adj_acoustic_accumulate<double, AccHost>>()},
    {"bc_periodic_x", runner<hx>()},
    {"bc_periodic_y", runner<hy>()},
    {"ppx_finish", runner<adj_ppx_finish<double, AccHost>>()},
    {"acoustic_w_solve", runner<adj_acoustic_w_solve<double, AccHost>>()},
};

template <void (*Fn)(const AdjArgs<float> &, int, int, int)>
void loop32(const AdjArgs<float> &A) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int tz = 0; tz < A.gz; tz++)
    for (int ty = 0; ty < A.gy; ty++)
      for (int tx = 0; tx < A.gx; tx++) Fn(A, tx, ty, tz);
}


typedef void (*Runner32)(const AdjArgs<float> &);

template <void (*Fn)(const AdjArgs<float> &, int, int, int)>
Runner32 runner32() {
  return loop32<Fn>;
}

void fx32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_lin_h<float, AccHost>(A, x, y, z, 0); }
void fy32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_lin_h<float, AccHost>(A, x, y, z, 1); }
void sx32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_stag_h<float, AccHost>(A, x, y, z, 0); }
void sy32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_stag_h<float, AccHost>(A, x, y, z, 1); }
void wx32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_weno_h<float, AccHost>(A, x, y, z, 0); }
void wy32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_weno_h<float, AccHost>(A, x, y, z, 1); }
void uvx32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_weno_uv_h<float, AccHost>(A, x, y, z, 0); }
void uvy32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_weno_uv_h<float, AccHost>(A, x, y, z, 1); }
void wwx32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_weno_w_h<float, AccHost>(A, x, y, z, 0); }
void wwy32(const AdjArgs<float> &A, int x, int y, int z) { adj_flux_weno_w_h<float, AccHost>(A, x, y, z, 1); }
void hx32(const AdjArgs<float> &A, int x, int y, int z) { adj_bc_periodic<float, AccHost>(A, x, y, z, 0); }
void hy32(const AdjArgs<float> &A, int x, int y, int z) { adj_bc_periodic<float, AccHost>(A, x, y, z, 1); }

struct Entry32 {
  const char *name;
  Runner32 run;
};

const Entry32 kTable32[] = {
    {"adv_flux_x", runner32<fx32>()},
    {"adv_flux_y", runner32<fy32>()},
    {"adv_flux_z", runner32<adj_flux_lin_z<float, AccHost>>()},
    {"adv_flux_x_stag", runner32<sx32>()},
    {"adv_flux_y_stag", runner32<sy32>()},
    {"adv_flux_z_stag", runner32<adj_flux_stag_z<float, AccHost>>()},
    {"adv_flux_x_weno", runner32<wx32>()},
    {"adv_flux_y_weno", runner32<wy32>()},
    {"adv_flux_z_weno", runner32<adj_flux_weno_z<float, AccHost>>()},
    {"adv_flux_x_weno_uv", runner32<uvx32>()},
    {"adv_flux_y_weno_uv", runner32<uvy32>()},
    {"adv_flux_z_weno_uv", runner32<adj_flux_weno_uv_z<float, AccHost>>()},
    {"adv_flux_x_weno_w", runner32<wwx32>()},
    {"adv_flux_y_weno_w", runner32<wwy32>()},
    {"adv_flux_z_weno_w", runner32<adj_flux_weno_w_z<float, AccHost>>()},
    {"adv_assemble", runner32<adj_assemble<float, AccHost>>()},
    {"rk_update", runner32<adj_rk_update<float, AccHost>>()},
    {"apply_thterm", runner32<adj_apply_thterm<float, AccHost>>()},
    {"buoyancy_apply", runner32<adj_buoyancy_apply<float, AccHost>>()},
    {"update_diagnostics_moist", runner32<adj_update_diagnostics_moist<float, AccHost>>()},
    {"stage_tendency_reset", runner32<adj_stage_tendency_reset<float, AccHost>>()},
    {"massflux_from_state", runner32<adj_massflux_from_state<float, AccHost>>()},
    {"div_massflux", runner32<adj_div_massflux<float, AccHost>>()},
    {"divergence3d", runner32<adj_divergence3d<float, AccHost>>()},
    {"velocity_to_massflux", runner32<adj_velocity_to_massflux<float, AccHost>>()},
    {"build_sadv", runner32<adj_build_sadv<float, AccHost>>()},
    {"stage_state_reset", runner32<adj_stage_state_reset<float, AccHost>>()},
    {"acoustic_begin", runner32<adj_acoustic_begin<float, AccHost>>()},
    {"acoustic_prepare", runner32<adj_acoustic_prepare<float, AccHost>>()},
    {"acoustic_uv", runner32<adj_acoustic_uv<float, AccHost>>()},
    {"acoustic_fpk", runner32<adj_acoustic_fpk<float, AccHost>>()},
    {"acoustic_pp", runner32<adj_acoustic_pp<float, AccHost>>()},
    {"acoustic_accumulate", runner32<adj_acoustic_accumulate<float, AccHost>>()},
    {"bc_periodic_x", runner32<hx32>()},
    {"bc_periodic_y", runner32<hy32>()},
    {"ppx_finish", runner32<adj_ppx_finish<float, AccHost>>()},
    {"acoustic_w_solve", runner32<adj_acoustic_w_solve<float, AccHost>>()},
};

}  // namespace

template <class R>
static void decode(AdjArgs<R> &A, const uint32_t *M, R *D, R *L, const uint32_t *ARG, uint64_t ptr_mask, int acoustic) {
  std::memset(&A, 0, sizeof A);
  A.gx = (int)ARG[0];
  A.gy = (int)ARG[1];
  A.gz = (int)ARG[2];
  const uint32_t g0 = ARG[4];
  A.g.nx = (int)M[g0];
  A.g.ny = (int)M[g0 + 1];
  A.g.nz = (int)M[g0 + 2];
  A.g.sJ = (int)M[g0 + 3];
  A.g.sK = (int)M[g0 + 4];
  A.g.rdx = wordf(M[g0 + 5]);
  A.g.rdy = wordf(M[g0 + 6]);
  A.g.rdz = wordf(M[g0 + 7]);
  if (acoustic) {
    const uint32_t a0 = ARG[5];
    A.a.dts = wordf(M[a0]);
    A.a.alph = wordf(M[a0 + 1]);
    A.a.beta = wordf(M[a0 + 2]);
    A.a.kdiv = wordf(M[a0 + 3]);
    A.a.smeps = wordf(M[a0 + 4]);
  }
  for (int n = 1; n < kMaxBindA; n++) {
    const uint32_t off = ARG[4 + n];
    if (ptr_mask >> n & 1u) {
      A.p[n] = D + off;
      A.l[n] = L + off;
    } else if (!(acoustic && n == 1)) {
      A.f[n] = wordf(M[off]);
      A.iv[n] = (int)M[off];
      A.iv2[n] = (int)M[off + 1];
    }
  }
}

extern "C" {

int teadj_has(const char *name) {
  for (const Entry &e : kTable)
    if (!std::strcmp(e.name, name)) return 1;
  return 0;
}

/* the binary32 instantiation (test infrastructure: the GPU's arithmetic on the host, over
 * the binary32 memory itself): values are the words of M read as floats */
int teadj_run32(const char *name, uint32_t *M, float *L, const uint32_t *ARG, uint64_t ptr_mask, int acoustic) {
  Runner32 run = nullptr;
  for (const Entry32 &e : kTable32)
    if (!std::strcmp(e.name, name)) run = e.run;
  if (!run) return -1;
  AdjArgs<float> A;
  decode<float>(A, M, reinterpret_cast<float *>(M), L, ARG, ptr_mask, acoustic);
  run(A);
  return 0;
}

int teadj_run(const char *name, const uint32_t *M, double *D, double *L, const uint32_t *ARG, uint64_t ptr_mask,
              int acoustic) {
  Runner run = nullptr;
  for (const Entry &e : kTable)
    if (!std::strcmp(e.name, name)) run = e.run;
  if (!run) return -1;
  AdjArgs<double> A;
  decode<double>(A, M, D, L, ARG, ptr_mask, acoustic);
  run(A);
  return 0;
}

}  // extern "C"

