// libocfd_gpu.so -- C ABI of the B200 (sm_100a) OpenCFD-Comb hot path (include/ocfd_gpu.h).
//
// Host side: parameter derivation (set_parameters, OCFD_readpara.f90:347-431), one device arena,
// the per-stage launch sequence of flow_time_advance (OCFD_Time_Adv.f90:7-92), Strang step
// capture into a CUDA graph, status words read back after every call, per-kernel event timing.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <array>
#include <cstring>
#include <map>
#include <stdexcept>
#include <utility>
#include <string>
#include <vector>

#define OCFD_DEFINE_CONST
#include "ocfd_chem.cuh"
#include "ocfd_device.cuh"
#include "ocfd_flow.cuh"
#include "ocfd_post.cuh"

namespace ocfd {
// the surrogate's flow-cell chemistry (ocfd_surrogate.cu)
int sg_cells_chem(int ns, double* f, double* Et, double* T, double* p, double* di, double dt2, int nsub, int* nfail,
                  cudaStream_t st);
int sg_cells_setup(int ns, long long N, double tol);
long long sg_cells_rejected(long long* reasons);
int sg_device_error(cudaStream_t st);
// set-up kernels (defined below) that the tile autotuner also launches
__global__ void k_fill(double* p, long long n, double v);
__global__ void k_jacobian(const double* X, const double* Y, const double* Z, double* const* m);
__global__ void k_metric_ratio(double* const* m, long long H);
// the wall-disturbance time of the next step of a multi-step run: ht = seq[counter++] (one thread;
// the steps of a run are ordered on one stream, so the counter needs no atomics)
__global__ void k_next_ht(const double* seq, int* counter, double* ht) {
  const int c = *counter;
  *ht = seq[c];
  *counter = c + 1;
}
}  // namespace ocfd
#include "ocfd_launch.h"

using namespace ocfd;

namespace {

std::string g_err;

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& s, int c) : std::runtime_error(s), code(c) {}
};
#define CK(x)                                                                                      \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess)                                                                         \
      throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_), OCFD_ERR_CUDA);             \
  } while (0)
#define LAUNCH_CHECK() CK(cudaGetLastError())

// kernel classes for event timing
// (species work of N_SPEC > 1, by kernel family: transport = k_transport, species_flux = the
// scalar k_flux sweeps, species_visc = k_ci + k_scal_ev + k_scal_div, species_rk = k_scal_rk)
enum KClass { KC_FLUX_X = 0, KC_FLUX_Y, KC_FLUX_Z, KC_VISC_EV, KC_VISC_DIV, KC_RK_PRIMS, KC_EXCH, KC_BC, KC_SENSOR,
              KC_TRANSPORT, KC_SPECIES_FLUX, KC_SPECIES_VISC, KC_SPECIES_RK, KC_CHEM, KC_OTHER, KC_NUM };
const char* kc_names[KC_NUM] = {"flux_x", "flux_y", "flux_z", "visc_ev", "visc_div", "rk_prims", "exchange",
                                "bc", "sensor", "transport", "species_flux", "species_visc", "species_rk",
                                "chem", "other"};

struct Lib {
  ocfd_params P{};
  DevConst hc{};
  int NS = 1;
  bool sep = false, have_kin = false, flow_ready = false;
  bool mech_on = true;  // run the compiled mechanism kernels when the loaded mechanism matches
  cudaStream_t st = nullptr;
  char* arena = nullptr;
  size_t arena_size = 0, arena_used = 0;
  double *f = nullptr, *fn = nullptr, *du = nullptr, *d = nullptr, *u = nullptr, *v = nullptr, *w = nullptr,
         *T = nullptr, *p = nullptr, *Et[2] = {nullptr, nullptr}, *di = nullptr, *din = nullptr, *Rh = nullptr;
  double *ev[12] = {}, *amu = nullptr, *amk = nullptr, *amd = nullptr, *qp[3] = {}, *ci = nullptr, *se[3] = {};
  double* dus = nullptr;  // Dus of every species (Ns x N)
  int chem_mode = 0;      // 0: FP64 integrator, 1: gated surrogate (ocfd_gpu_chem_mode)
  int g_mode = -1;        // chemistry mode of the captured graph
  double *X = nullptr, *Y = nullptr, *Z = nullptr, *met[19] = {}, *d1[3] = {}, *edge[6] = {}, *partial = nullptr;
  double *inlet = nullptr, *upper = nullptr, *wall = nullptr, *ht_dev = nullptr;
  int *nonref = nullptr, *patches = nullptr;
  int npatch = 0;
  DevStatus* sdev = nullptr;
  DevStatus* shost = nullptr;
  double* ht_host = nullptr;
  int cur = 0;  // which Et buffer is current
  Geo geo{};
  int inlet_kind = 0, upper_kind = 0, outlet = 0;
  std::vector<double> tm, fait;
  // graph of one Strang step (the captured graph is kept as the child of the chunk graph, which
  // replays RUN_CHUNK steps with one launch)
  cudaGraphExec_t gexec = nullptr, gchunk = nullptr;
  // second stream of a stage: k_visc_ev and its halo exchange run beside the flux sweeps
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // third stream of a stage with species (N_SPEC > 1): the species sweeps, the species viscous
  // divergence and the species RK update run beside the transport, Qp and flow kernels
  cudaStream_t st3 = nullptr;
  cudaEvent_t ev_sp_fork = nullptr, ev_se_done = nullptr, ev_sp_join = nullptr;
  bool fork_species = true;
  bool fork_visc = true;
  cudaGraph_t gstep = nullptr;
  int* ht_counter = nullptr;
  double g_dt = 0;
  int g_ifr = -1, g_nsub = -1, g_par = -1, g_launches = 0;
  // stencil tile choices (ocfd_gpu_set_tiles / ocfd_gpu_autotune): flow-flux tile shape per
  // sweep direction, k planes per block of k_visc_ev and k_visc_div
  int flux_ts[3] = {0, 0, 0};
  int kc_ev = VE_KC, kc_div = VE_KC;
  // metric form per kernel family on a tensor-product grid: false = computed from the 1-D
  // derivatives (separable), true = read from the 19 stored arrays (allocated on first use)
  bool met_flux = false, met_ev = false, met_div = false;
  double* met_store = nullptr;
  // analysis (ocfd_gpu_keep_viscosity, ocfd_gpu_ana_*): the single-species stage viscosity kept
  // for ana_box, reduction partials, time-average accumulators
  bool keep_amu = false;
  double *amu_keep = nullptr, *ana_part = nullptr, *avg = nullptr;
  size_t ana_part_n = 0;
  int k_average = 0;
  double t_average = 0.0;
  // asynchronous save / show (ocfd_gpu_snapshot*, ocfd_gpu_diag_begin/end): a copy stream, two
  // snapshot slots (device pack buffer + pinned host buffer; state 0 free, 1 in flight or
  // unread, 2 handed out), the show_flow_msg sums
  cudaStream_t cst = nullptr;
  double *snap_dev[2] = {}, *snap_host[2] = {};
  cudaEvent_t snap_ready[2] = {}, snap_done[2] = {};
  int snap_state[2] = {0, 0}, snap_istep[2] = {0, 0};
  double snap_tt[2] = {0.0, 0.0};
  long long snap_seq[2] = {0, 0}, snap_counter = 0;
  double *diag_dev = nullptr, *diag_host = nullptr;
  cudaEvent_t diag_ready = nullptr, diag_done = nullptr;
  bool diag_pending = false;
  // batched chemistry scratch
  double *b_di = nullptr, *b_e = nullptr, *b_dt = nullptr;
  int *b_nsub = nullptr, *b_perm = nullptr, *b_hist = nullptr, *b_counter = nullptr, *b_nfail = nullptr;
  size_t b_cap = 0;
  int b_last[2] = {0, 0};  // the last batch call's Newton non-convergences and bad reactors
  // profiling
  bool prof = false;
  double kc_ms[KC_NUM] = {};
  long long kc_n[KC_NUM] = {};
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  std::vector<std::pair<int, int>> ev_pending;  // (class, pool index)
  long long launches = 0;
  // bench support
  cudaEvent_t uev[16] = {};
  double* ht_seq = nullptr;
  double* ht_seq_host = nullptr;
  int ht_cap = 0;
};
Lib* L = nullptr;

template <class T>
T* alloc(size_t n) {
  size_t bytes = (n * sizeof(T) + 255) & ~(size_t)255;
  if (L->arena_used + bytes > L->arena_size) throw std::runtime_error("device arena exhausted");
  T* p = reinterpret_cast<T*>(L->arena + L->arena_used);
  L->arena_used += bytes;
  return p;
}

// ---------------------------------------------------------------- launch helpers
struct KTimer {
  int cls;
  int idx = -1;
  KTimer(int c) : cls(c) {
    L->launches++;
    if (!L->prof) return;
    if (L->ev_pending.size() >= L->ev_pool.size()) {
      cudaEvent_t a, b;
      CK(cudaEventCreate(&a));
      CK(cudaEventCreate(&b));
      L->ev_pool.push_back({a, b});
    }
    idx = (int)L->ev_pending.size();
    CK(cudaEventRecord(L->ev_pool[idx].first, L->st));
  }
  ~KTimer() noexcept(false) {
    if (idx < 0) return;
    CK(cudaEventRecord(L->ev_pool[idx].second, L->st));
    L->ev_pending.push_back({cls, idx});
  }
};
void prof_collect() {
  if (L->ev_pending.empty()) return;
  CK(cudaStreamSynchronize(L->st));
  for (auto& pr : L->ev_pending) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, L->ev_pool[pr.second].first, L->ev_pool[pr.second].second));
    L->kc_ms[pr.first] += ms;
    L->kc_n[pr.first] += 1;
  }
  L->ev_pending.clear();
}

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

void exchange(std::initializer_list<double*> fields, int dirmask) {
  ExchArgs a{};
  a.nf = 0;
  for (double* f : fields) a.f[a.nf++] = f;
  a.dirmask = dirmask;
  bool any = false;
  for (int dd = 0; dd < 3; dd++)
    if ((dirmask >> dd & 1) && L->P.iperiodic[dd]) any = true;
  if (!any || a.nf == 0) return;
  const int nx = L->P.nx, ny = L->P.ny, nz = L->P.nz;
  long long mx = std::max((long long)ny * nz, std::max((long long)nx * nz, (long long)nx * ny)) * OCFD_L;
  KTimer t(KC_EXCH);
  k_exchange<<<dim3(nblk(mx, 256), a.nf), 256, 0, L->st>>>(a);
  LAUNCH_CHECK();
}
void exchange_v(const std::vector<double*>& fields, int dirmask) {
  for (size_t s = 0; s < fields.size(); s += 24) {
    ExchArgs a{};
    a.nf = 0;
    for (size_t m = s; m < fields.size() && m < s + 24; m++) a.f[a.nf++] = fields[m];
    a.dirmask = dirmask;
    const int nx = L->P.nx, ny = L->P.ny, nz = L->P.nz;
    long long mx = std::max((long long)ny * nz, std::max((long long)nx * nz, (long long)nx * ny)) * OCFD_L;
    KTimer t(KC_EXCH);
    k_exchange<<<dim3(nblk(mx, 256), a.nf), 256, 0, L->st>>>(a);
    LAUNCH_CHECK();
  }
}

// ---- flux dispatch (kernels compiled in ocfd_flux_{x,y,z}.cu) ----
// group = 0: the flow fluxes; else a scalar sweep of every species, group species per block
void launch_flux(int dir, const FluxArgs& a, int group = 0, int ngroups = 1) {
  KTimer t(group ? KC_SPECIES_FLUX : KC_FLUX_X + dir);
  const ocfd_params& P = L->P;
  const bool ch = P.if_scheme_character == 1;
  const int ts = (group == 0 && !ch) ? L->flux_ts[dir] : 0;
  const bool sep = L->sep && !L->met_flux;
  if (ts != 0) {
    using Fn = void (*)(int, int, bool, const FluxArgs&, int, int, int, cudaStream_t);
    static const Fn tab[3][2] = {{launch_flux_x_t1, launch_flux_x_t2},
                                 {launch_flux_y_t1, launch_flux_y_t2},
                                 {launch_flux_z_t1, launch_flux_z_t2}};
    tab[dir][ts - 1](P.scheme_invis, P.flux_splitting, sep, a, P.nx, P.ny, P.nz, L->st);
  } else if (dir == 0) launch_flux_x(P.scheme_invis, P.flux_splitting, sep, group, ngroups, ch, a, P.nx, P.ny, P.nz, L->st);
  else if (dir == 1) launch_flux_y(P.scheme_invis, P.flux_splitting, sep, group, ngroups, ch, a, P.nx, P.ny, P.nz, L->st);
  else launch_flux_z(P.scheme_invis, P.flux_splitting, sep, group, ngroups, ch, a, P.nx, P.ny, P.nz, L->st);
  LAUNCH_CHECK();
}

// NS dispatch for the species-templated kernels (N_SPEC 1, 2 and 9 always; 3..8 unless
// OCFD_FEW_SPECIES is defined, which shortens development builds)
#ifdef OCFD_FEW_SPECIES
#define NS_MORE(...)
#else
#define NS_MORE(...)                                               \
    case 3: { constexpr int NSV = 3; __VA_ARGS__; } break;          \
    case 4: { constexpr int NSV = 4; __VA_ARGS__; } break;          \
    case 5: { constexpr int NSV = 5; __VA_ARGS__; } break;          \
    case 6: { constexpr int NSV = 6; __VA_ARGS__; } break;          \
    case 7: { constexpr int NSV = 7; __VA_ARGS__; } break;          \
    case 8: { constexpr int NSV = 8; __VA_ARGS__; } break;
#endif
#define NS_DISPATCH(ns, ...)                                  \
  switch (ns) {                                                \
    case 1: { constexpr int NSV = 1; __VA_ARGS__; } break;            \
    case 2: { constexpr int NSV = 2; __VA_ARGS__; } break;            \
    NS_MORE(__VA_ARGS__)                                       \
    case 9: { constexpr int NSV = 9; __VA_ARGS__; } break;            \
    default: throw std::runtime_error("N_SPEC must be 1..9"); \
  }

// ---------------------------------------------------------------- stages
BcArgs bc_args() {
  BcArgs a{};
  a.f = L->f; a.d = L->d; a.u = L->u; a.v = L->v; a.w = L->w; a.T = L->T; a.p = L->p; a.Et = L->Et[L->cur];
  a.di = L->di;
  a.inlet = L->inlet; a.upper = L->upper; a.wall_pertb = L->wall; a.nonref = L->nonref;
  a.inlet_kind = L->inlet_kind; a.upper_kind = L->upper_kind; a.outlet = L->outlet;
  a.jet_iflag = (int)std::lround(L->P.bc_para[0]);
  a.Tw = L->P.bc_para[4]; a.xinit = L->P.bc_para[5]; a.disA = L->P.bc_para[7];
  a.ht = 0.0;
  a.X = L->X;
  a.g = L->geo;
  return a;
}

template <int NS>
void ocfd_bc_t() {
  BcArgs a = bc_args();
  const int nx = L->P.nx, ny = L->P.ny, nz = L->P.nz;
  if (L->P.ibc == OCFD_BC_BOUNDARYLAYER) {
    KTimer t(KC_BC);
    k_bc_inlet<NS><<<nblk((long long)ny * nz, 128), 128, 0, L->st>>>(a);
    LAUNCH_CHECK();
    if (L->upper_kind >= 0) {
      k_bc_upper<NS><<<nblk((long long)nx * nz, 128), 128, 0, L->st>>>(a);
      LAUNCH_CHECK();
    }
  }
  if (L->P.ibc == OCFD_BC_BOUNDARYLAYER) {
    KTimer t(KC_BC);
    // the wall disturbance amplitude h(t) is read from device memory so that a captured graph
    // picks up the current step's value
    a.ht = 0.0;
    if (L->sep) k_bc_wall<NS, true><<<nblk((long long)nx * nz, 128), 128, 0, L->st>>>(a, L->ht_dev);
    else k_bc_wall<NS, false><<<nblk((long long)nx * nz, 128), 128, 0, L->st>>>(a, L->ht_dev);
    LAUNCH_CHECK();
    if (L->outlet == 1 || L->outlet == 2) {
      k_bc_outlet<NS><<<nblk((long long)ny * nz, 128), 128, 0, L->st>>>(a);
      LAUNCH_CHECK();
    }
  }
  if (L->P.ibc == OCFD_BC_JET) {
    KTimer t(KC_BC);
    k_bc_jet_inlet<NS><<<nblk((long long)ny * nz, 128), 128, 0, L->st>>>(a);
    LAUNCH_CHECK();
    k_bc_jet_outlet<NS><<<nblk((long long)ny * nz, 128), 128, 0, L->st>>>(a);
    LAUNCH_CHECK();
  }
  {
    KTimer t(KC_BC);
    k_bc_faces<NS><<<nblk(2LL * ny * nz, 128), 128, 0, L->st>>>(a, 0);
    LAUNCH_CHECK();
    k_bc_faces<NS><<<nblk(2LL * (nx - 2) * nz, 128), 128, 0, L->st>>>(a, 1);
    LAUNCH_CHECK();
    k_bc_faces<NS><<<nblk(2LL * (nx - 2) * (ny - 2), 128), 128, 0, L->st>>>(a, 2);
    LAUNCH_CHECK();
  }
  for (int face = 0; face < 6; face++) {
    if (!(L->P.ghost_cell[face] == 1 || L->P.ghost_cell[face] == 2)) continue;
    int dir = face / 2;
    long long na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
    KTimer t(KC_BC);
    k_bc_ghost<NS><<<nblk(na * nb * OCFD_L, 128), 128, 0, L->st>>>(a, face);
    LAUNCH_CHECK();
  }
}

template <int NS>
void prims_t(int krk, double dt) {
  PrimArgs a{};
  a.f = L->f; a.fn = L->fn; a.du = L->du;
  a.d = L->d; a.u = L->u; a.v = L->v; a.w = L->w; a.T = L->T; a.p = L->p;
  a.Et = L->Et[1 - L->cur];
  a.di = L->di;
  a.st = L->sdev;
  a.krk = krk;
  a.dt = dt;
  {
    KTimer t(KC_RK_PRIMS);
    const unsigned nb = nblk(L->hc.N, 256);
    switch (krk) {
      case 1: k_rk_prims<NS, 1><<<nb, 256, 0, L->st>>>(a); break;
      case 2: k_rk_prims<NS, 2><<<nb, 256, 0, L->st>>>(a); break;
      case 3: k_rk_prims<NS, 3><<<nb, 256, 0, L->st>>>(a); break;
      default: k_rk_prims<NS, 0><<<nb, 256, 0, L->st>>>(a); break;
    }
    LAUNCH_CHECK();
  }
  {
    KTimer t(KC_OTHER);
    k_repair_et<NS><<<1, 32, 0, L->st>>>(L->f, L->Et[1 - L->cur], L->Et[L->cur], L->T, L->p, L->di, L->sdev);
    LAUNCH_CHECK();
  }
  L->cur = 1 - L->cur;
}

void sensor() {
  int sensor = (int)std::lround(L->P.hybrid_para[0]);
  long long N = L->hc.N;
  KTimer t(KC_SENSOR);
  if (sensor == 1) {
    k_sensor1<<<nblk(N, 256), 256, 0, L->st>>>(L->p, L->Rh, L->npatch, L->patches);
    LAUNCH_CHECK();
  } else {
    unsigned nb = nblk(N, 256);
    if (L->sep) k_sensor2<true><<<nb, 256, 0, L->st>>>(L->p, L->Rh, L->partial, L->geo);
    else k_sensor2<false><<<nb, 256, 0, L->st>>>(L->p, L->Rh, L->partial, L->geo);
    LAUNCH_CHECK();
    k_sensor2_scale<<<nb, 256, 0, L->st>>>(L->Rh, L->partial, (int)nb, L->npatch, L->patches);
    LAUNCH_CHECK();
  }
}

// k_visc_ev over (i, j) tiles and k chunks; HZ = the CD6 / CD8 stencil half-width
template <int NS, bool SEP, int HZ>
void visc_ev_go(const ViscArgs& va) {
  constexpr size_t sm = VeTile<HZ>::smem;
  static bool attr = false;
  if (!attr) {
    CK(cudaFuncSetAttribute(k_visc_ev<NS, SEP, HZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  const ocfd_params& P = L->P;
  dim3 grid(nblk(P.nx, VE_TX), nblk(P.ny, VE_TY), nblk(P.nz, va.kc));
  k_visc_ev<NS, SEP, HZ><<<grid, VE_THREADS, sm, L->st>>>(va);
}

template <bool SEP, int HZ>
void visc_div_go(const DivArgs& da) {
  constexpr size_t sm = VdTile<HZ>::smem;
  static bool attr = false;
  if (!attr) {
    CK(cudaFuncSetAttribute(k_visc_div<SEP, HZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  const ocfd_params& P = L->P;
  if (da.kc == 0) {  // per-cell form
    k_visc_div_pc<SEP, HZ><<<nblk(L->hc.N, 256), 256, 0, L->st>>>(da);
    return;
  }
  dim3 grid(nblk(P.nx, VE_TX), nblk(P.ny, VE_TY), nblk(P.nz, da.kc));
  k_visc_div<SEP, HZ><<<grid, VE_THREADS, sm, L->st>>>(da);
}

// kernel arguments of the stage's flow sweeps and viscous kernels on the current state
FluxArgs flow_flux_args() {
  FluxArgs fa{};
  fa.d = L->d; fa.u = L->u; fa.v = L->v; fa.w = L->w; fa.p = L->p; fa.Et = L->Et[L->cur]; fa.Rh = L->Rh;
  fa.out = L->du;
  fa.g = L->geo;
  return fa;
}
template <int NS>
ViscArgs visc_args() {
  ViscArgs va{};
  va.d = L->d; va.u = L->u; va.v = L->v; va.w = L->w; va.T = L->T; va.di = L->di;
  if (NS > 1) {
    va.amu = L->amu; va.amk = L->amk;
    va.qpx = L->qp[0]; va.qpy = L->qp[1]; va.qpz = L->qp[2];
  }
  for (int dd = 0; dd < 3; dd++)
    for (int m = 0; m < 4; m++) va.ev[dd][m] = L->ev[4 * dd + m];
  va.g = L->geo;
  va.kc = L->kc_ev;
  return va;
}
DivArgs div_args() {
  DivArgs da{};
  for (int m = 0; m < 12; m++) da.ev[m] = L->ev[m];
  da.du = L->du;
  da.g = L->geo;
  da.kc = L->kc_div;
  return da;
}
template <int NS>
void visc_ev_launch(const ViscArgs& va) {
  const bool cd8 = L->P.scheme_vis == OCFD_SCHEME_CD8;
  if (L->sep && !L->met_ev) cd8 ? visc_ev_go<NS, true, 4>(va) : visc_ev_go<NS, true, 3>(va);
  else cd8 ? visc_ev_go<NS, false, 4>(va) : visc_ev_go<NS, false, 3>(va);
  LAUNCH_CHECK();
}
void visc_div_launch(const DivArgs& da) {
  const bool cd8 = L->P.scheme_vis == OCFD_SCHEME_CD8;
  if (L->sep && !L->met_div) cd8 ? visc_div_go<true, 4>(da) : visc_div_go<true, 3>(da);
  else cd8 ? visc_div_go<false, 4>(da) : visc_div_go<false, 3>(da);
  LAUNCH_CHECK();
}

// the flow part of a stage's right-hand side: the three flux sweeps into du, the viscous fluxes
// Ev with their halo exchange, and their divergence added to du
template <int NS>
void flow_rhs_t(const FluxArgs& fa) {
  const bool visc = L->P.if_viscous == 1;
  auto visc_ev_part = [&]() {
    {
      KTimer t(KC_VISC_EV);
      visc_ev_launch<NS>(visc_args<NS>());
    }
    exchange({L->ev[0], L->ev[1], L->ev[2], L->ev[3]}, 1);
    exchange({L->ev[4], L->ev[5], L->ev[6], L->ev[7]}, 2);
    exchange({L->ev[8], L->ev[9], L->ev[10], L->ev[11]}, 4);
  };
  // k_visc_ev reads only the primitives (and, for N_SPEC > 1, the transport and enthalpy fluxes
  // computed above) and writes only Ev, while the flux sweeps write du: the two run side by side
  // on two streams (two branches of the step's graph), joined before k_visc_div. The per-kernel
  // timing mode keeps them in order.
  const bool fork = visc && L->fork_visc && !L->prof && L->st2;
  if (fork) {
    CK(cudaEventRecord(L->ev_fork, L->st));
    CK(cudaStreamWaitEvent(L->st2, L->ev_fork, 0));
    std::swap(L->st, L->st2);  // the launch helpers use L->st
    try {
      visc_ev_part();
    } catch (...) {
      std::swap(L->st, L->st2);
      throw;
    }
    CK(cudaEventRecord(L->ev_join, L->st));
    std::swap(L->st, L->st2);
  }
  for (int dd = 0; dd < 3; dd++) launch_flux(dd, fa);
  if (visc) {
    if (fork) CK(cudaStreamWaitEvent(L->st, L->ev_join, 0));
    else visc_ev_part();
    {
      KTimer t(KC_VISC_DIV);
      visc_div_launch(div_args());
    }
  }
}

template <int NS>
void stage_rhs_t(int krk, double dt1, bool rk);

template <int NS>
void stage_t(int krk, double dt1) {
  const long long N = L->hc.N, H = L->hc.H;
  double* Etc = L->Et[L->cur];
  if (NS == 1 && L->keep_amu) {  // comput_Amu_Amk_AMD's Amu at the stage start, for ana_box
    KTimer t(KC_OTHER);
    k_amu1<<<nblk(N, 256), 256, 0, L->st>>>(L->T, L->di, L->amu_keep);
    LAUNCH_CHECK();
  }
  if (NS > 1) {
    KTimer t(KC_TRANSPORT);
    k_transport<NS><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->d, L->T, L->p, L->di, L->amu, L->amk, L->amd);
    LAUNCH_CHECK();
  }
  {
    std::vector<double*> fl = {L->d, L->u, L->v, L->w, L->T, L->p, Etc};
    if (NS > 1)
      for (int m = 0; m < NS; m++) fl.push_back(L->di + (size_t)m * H);
    exchange_v(fl, 7);
  }
  if (krk == 1 && L->P.scheme_invis == OCFD_SCHEME_HYBRID) {
    sensor();
    exchange({L->Rh}, 7);
  }
  stage_rhs_t<NS>(krk, dt1, true);
  // N_SPEC = 1: di = d over the whole array (OCFD_Time_Adv.f90:45-52). Nothing between the stage
  // start and here reads di, and the inline transport of k_visc_ev must see the previous stage's
  // di (comput_Amu_Amk_AMD runs before the copy in the reference), so the copy happens here.
  if (NS == 1) {
    KTimer t(KC_EXCH);
    k_copy<<<nblk(H, 256), 256, 0, L->st>>>(L->d, L->di, H);
    LAUNCH_CHECK();
  }
  prims_t<NS>(krk, dt1);
  ocfd_bc_t<NS>();
}

// The right-hand sides of a stage: the species (inviscid sweeps, viscous fluxes and their
// divergence, and with rk the species RK update) and the flow (flow_rhs_t). Without rk it writes
// only arrays that every stage recomputes before reading them (Dus, ci, the species viscous
// fluxes, Qp, du, Ev), which the tuner uses to time it on the current state.
template <int NS>
void stage_rhs_t(int krk, double dt1, bool rk) {
  const long long N = L->hc.N, H = L->hc.H;
  FluxArgs fa = flow_flux_args();
  // Species (every species at once: du_scaler_invis / du_scaler_viscous / Scalar_time_adv_RK3 of
  // the reference's species loop; Dus of species m is dus + m N). The species sweeps read only di
  // and the velocities and write only Dus, and nothing of the flow part reads di, so the sweeps,
  // the species divergence (after the species viscous fluxes) and the species RK update run on a
  // third stream beside k_ci / k_scal_ev and the flow part (branches of the step's graph), joined
  // before k_rk_prims, which reads the updated di. Each kernel writes what it wrote before, so the
  // results do not depend on the overlap. The per-kernel timing mode keeps everything in order.
  const bool spfork = NS > 1 && L->fork_species && !L->prof && L->st3;
  auto on_st3 = [&](auto&& body) {  // launches of body go to the third stream
    std::swap(L->st, L->st3);
    try {
      body();
    } catch (...) {
      std::swap(L->st, L->st3);
      throw;
    }
    std::swap(L->st, L->st3);
  };
  const bool sp_visc = NS > 1 && L->P.if_viscous == 1;
  auto species_sweeps = [&]() {
    const int grp = NS % 3 == 0 ? 3 : 1;
    FluxArgs fs = fa;
    fs.fs = L->di;
    fs.out = L->dus;
    for (int dd = 0; dd < 3; dd++) launch_flux(dd, fs, grp, NS / grp);
  };
  auto species_div_rk = [&]() {
    if (sp_visc && rk) {  // the divergence with the species RK update fused in
      KTimer t(KC_SPECIES_VISC);
      if (L->sep)
        k_scal_div<NS, true, true><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->se[0], L->se[1], L->se[2], L->dus,
                                                                          L->geo, krk, dt1, L->din, L->di);
      else
        k_scal_div<NS, false, true><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->se[0], L->se[1], L->se[2], L->dus,
                                                                           L->geo, krk, dt1, L->din, L->di);
      LAUNCH_CHECK();
      return;
    }
    if (sp_visc) {
      KTimer t(KC_SPECIES_VISC);
      if (L->sep) k_scal_div<NS, true><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->se[0], L->se[1], L->se[2], L->dus, L->geo);
      else k_scal_div<NS, false><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->se[0], L->se[1], L->se[2], L->dus, L->geo);
      LAUNCH_CHECK();
    }
    if (rk) {
      KTimer t(KC_SPECIES_RK);
      k_scal_rk<<<dim3(nblk(N, 256), NS), 256, 0, L->st>>>(krk, dt1, L->dus, L->din, L->di);
      LAUNCH_CHECK();
    }
  };
  if (NS > 1) {
    if (spfork) {
      CK(cudaEventRecord(L->ev_sp_fork, L->st));
      CK(cudaStreamWaitEvent(L->st3, L->ev_sp_fork, 0));
      on_st3(species_sweeps);
    } else {
      species_sweeps();
    }
    if (sp_visc) {
      {
        KTimer t(KC_SPECIES_VISC);
        k_ci<<<dim3(nblk(H, 256), NS), 256, 0, L->st>>>(L->di, L->d, L->ci, H);
        LAUNCH_CHECK();
        if (L->sep) k_scal_ev<NS, true><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->ci, L->d, L->T, L->amd, L->qp[0], L->qp[1], L->qp[2], L->se[0], L->se[1], L->se[2], L->geo);
        else k_scal_ev<NS, false><<<nblk(N, 32), dim3(32, NS), 0, L->st>>>(L->ci, L->d, L->T, L->amd, L->qp[0], L->qp[1], L->qp[2], L->se[0], L->se[1], L->se[2], L->geo);
        LAUNCH_CHECK();
      }
      for (int dd = 0; dd < 3; dd++) {
        std::vector<double*> fl;
        for (int m = 0; m < NS; m++) fl.push_back(L->se[dd] + (size_t)m * H);
        exchange_v(fl, 1 << dd);
      }
    }
    if (spfork) {
      CK(cudaEventRecord(L->ev_se_done, L->st));
      on_st3([&]() {
        CK(cudaStreamWaitEvent(L->st, L->ev_se_done, 0));
        species_div_rk();
        CK(cudaEventRecord(L->ev_sp_join, L->st));
      });
    } else {
      species_div_rk();
    }
  }
  fa.fs = nullptr;
  fa.out = L->du;
  flow_rhs_t<NS>(fa);
  if (spfork) CK(cudaStreamWaitEvent(L->st, L->ev_sp_join, 0));
}

template <int NS>
void flow_advance_t(double dt1) {
  const long long N = L->hc.N, H = L->hc.H;
  CK(cudaMemcpyAsync(L->fn, L->f, sizeof(double) * 5 * N, cudaMemcpyDeviceToDevice, L->st));
  if (NS > 1) {
    // din <- di (interior only); a strided 3-D copy per species
    for (int m = 0; m < NS; m++) {
      cudaMemcpy3DParms cp{};
      cp.srcPtr = make_cudaPitchedPtr(L->di + (size_t)m * H + (OCFD_L + L->hc.HX * (OCFD_L + (long long)L->hc.HY * OCFD_L)),
                                      sizeof(double) * L->hc.HX, L->hc.HX, L->hc.HY);
      cp.dstPtr = make_cudaPitchedPtr(L->din + (size_t)m * N, sizeof(double) * L->P.nx, L->P.nx, L->P.ny);
      cp.extent = make_cudaExtent(sizeof(double) * L->P.nx, L->P.ny, L->P.nz);
      cp.kind = cudaMemcpyDeviceToDevice;
      CK(cudaMemcpy3DAsync(&cp, L->st));
    }
  }
  for (int krk = 1; krk <= 3; krk++) stage_t<NS>(krk, dt1);
}

template <int NS>
void chem_t(double dt2, int nsub) {
  KTimer t(KC_CHEM);
  if (L->chem_mode == 1) {
    const int rc = sg_cells_chem(NS, L->f, L->Et[L->cur], L->T, L->p, L->di, dt2, nsub, &L->sdev->newton_fail, L->st);
    if (rc == -5) throw std::runtime_error("surrogate chemistry not set up for this grid and mechanism");
    if (rc != 0) throw CudaError("surrogate chemistry: the network launch failed", OCFD_ERR_CUDA);
  } else {
    launch_chem_cells(NS, L->hc.N, L->f, L->Et[L->cur], L->T, L->p, L->di, dt2, nsub, &L->sdev->newton_fail, L->st);
  }
  LAUNCH_CHECK();
}

// ---------------------------------------------------------------- stencil tile autotuner
// Tile choices {flux x, y, z shape; k_visc_ev, k_visc_div k planes per block; metric form of the
// flux sweeps, k_visc_ev, k_visc_div; k_visc_ev beside the flux sweeps on a second stream or after
// them}. Every choice gives bit-identical results (a tile decides
// which block computes a point, not how; the stored metric arrays hold the values the separable
// form computes), so the tuner is free to pick by time alone. Choices are remembered per
// configuration in the process.
constexpr int TUNE_N = 9, TUNE_TIMES = 3 * FLUX_TILE_SHAPES + 9 + 5 + 2 + 2;
std::map<std::string, std::array<int, TUNE_N>> g_tune_cache;

std::string tune_key() {
  const ocfd_params& P = L->P;
  char b[200];
  std::snprintf(b, sizeof b, "%d %d %d|%d %d %d %d|%d %d %d", P.nx, P.ny, P.nz, P.scheme_invis, P.flux_splitting,
                P.if_scheme_character, (int)L->sep, L->NS, P.if_viscous, P.scheme_vis);
  return b;
}

void set_geo_device_ptrs();
// forgets the captured step and the chunk graph built on it (re-captured at the next step)
void drop_graphs() {
  if (L->gchunk) { CK(cudaGraphExecDestroy(L->gchunk)); L->gchunk = nullptr; }
  if (L->gexec) { CK(cudaGraphExecDestroy(L->gexec)); L->gexec = nullptr; }
  if (L->gstep) { CK(cudaGraphDestroy(L->gstep)); L->gstep = nullptr; }
}
// the 19 metric arrays of a tensor-product grid, as the general path computes them
// (comput_Jacobian3d, the periodic exchange, Akx1..Asz1), beside the separable form
void ensure_stored_metrics() {
  if (!L->sep || L->met_store) return;
  const long long H = L->hc.H, N = L->hc.N;
  CK(cudaMalloc(&L->met_store, sizeof(double) * 19 * H));
  for (int m = 0; m < 19; m++) L->met[m] = L->met_store + (size_t)m * H;
  for (int m = 0; m < 19; m++) {
    k_fill<<<nblk(H, 256), 256, 0, L->st>>>(L->met[m], H, 1.0);
    LAUNCH_CHECK();
  }
  double** mp = nullptr;
  CK(cudaMalloc(&mp, sizeof(double*) * 19));
  CK(cudaMemcpyAsync(mp, L->met, sizeof(double*) * 19, cudaMemcpyHostToDevice, L->st));
  k_jacobian<<<nblk(N, 256), 256, 0, L->st>>>(L->X, L->Y, L->Z, mp);
  LAUNCH_CHECK();
  std::vector<double*> ml(L->met, L->met + 10);
  exchange_v(ml, 7);
  k_metric_ratio<<<nblk(H, 256), 256, 0, L->st>>>(mp, H);
  LAUNCH_CHECK();
  CK(cudaStreamSynchronize(L->st));
  CK(cudaFree(mp));
  set_geo_device_ptrs();
}

void apply_tiles(const int* c) {
  for (int d = 0; d < 3; d++) L->flux_ts[d] = c[d];
  L->kc_ev = c[3];
  L->kc_div = c[4];
  if (L->sep && (c[5] | c[6] | c[7])) ensure_stored_metrics();
  L->met_flux = c[5] != 0;
  L->met_ev = c[6] != 0;
  L->met_div = c[7] != 0;
  L->fork_visc = (c[8] & 1) != 0;
  L->fork_species = (c[8] & 2) != 0;
  drop_graphs();  // the captured step holds the old launches
}

// times every candidate of each family on the current state (one warm-up launch, then reps
// launches between two events) and applies the fastest; the launches write only scratch arrays
// (du, Ev, the hybrid sensor) that every stage recomputes before it reads them
template <int NS>
void tune_t(int reps, int* best, double* ms) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto timed = [&](auto&& launch) {
    launch();
    CK(cudaEventRecord(e0, L->st));
    for (int r = 0; r < reps; r++) launch();
    CK(cudaEventRecord(e1, L->st));
    CK(cudaEventSynchronize(e1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e0, e1));
    return (double)t / reps;
  };
  try {
    const ocfd_params& P = L->P;
    if (P.scheme_invis == OCFD_SCHEME_HYBRID) {
      sensor();
      exchange({L->Rh}, 7);
    }
    const FluxArgs fa = flow_flux_args();
    const bool ch = P.if_scheme_character == 1;
    for (int d = 0; d < 3; d++) {
      double tmin = 1e300;
      best[d] = 0;
      for (int ts = 0; ts < FLUX_TILE_SHAPES; ts++) {
        if (ch && ts > 0) { ms[d * FLUX_TILE_SHAPES + ts] = -1.0; continue; }  // one characteristic tile
        L->flux_ts[d] = ts;
        const double t = timed([&] { launch_flux(d, fa); });
        ms[d * FLUX_TILE_SHAPES + ts] = t;
        if (t < tmin) { tmin = t; best[d] = ts; }
      }
      L->flux_ts[d] = best[d];
    }
    best[3] = best[4] = VE_KC;
    best[5] = best[6] = best[7] = L->sep ? 0 : 1;
    best[8] = NS > 1 ? 3 : 1;
    for (int m = 3 * FLUX_TILE_SHAPES; m < TUNE_TIMES; m++) ms[m] = -1.0;
    if (P.if_viscous == 1) {
      double t_ev = 1e300, t_div = 1e300;
      for (int m = 0; m < 4; m++) {
        ViscArgs va = visc_args<NS>();
        va.kc = VE_KC_CHOICES[m];
        const double t = timed([&] { visc_ev_launch<NS>(va); });
        ms[3 * FLUX_TILE_SHAPES + m] = t;
        if (t < t_ev) { t_ev = t; best[3] = va.kc; }
      }
      for (int m = 0; m < 5; m++) {  // the four k chunks, then the per-cell form (0)
        DivArgs da = div_args();
        da.kc = m < 4 ? VE_KC_CHOICES[m] : 0;
        const double t = timed([&] { visc_div_launch(da); });
        ms[3 * FLUX_TILE_SHAPES + 4 + m] = t;
        if (t < t_div) { t_div = t; best[4] = da.kc; }
      }
    }
    if (L->sep) {  // the stored metric arrays, each family at its best tile
      ensure_stored_metrics();
      const FluxArgs fm = flow_flux_args();  // geometry with the stored arrays
      const int M0 = 3 * FLUX_TILE_SHAPES + 9;
      L->met_flux = true;
      for (int d = 0; d < 3; d++) {
        L->flux_ts[d] = best[d];
        const double t = timed([&] { launch_flux(d, fm); });
        ms[M0 + d] = t;
        if (t < ms[d * FLUX_TILE_SHAPES + best[d]]) best[5] = 1;  // one form for the three sweeps
      }
      if (best[5] == 1) {  // keep the stored form only if the three sweeps together are faster
        double a = 0.0, b = 0.0;
        for (int d = 0; d < 3; d++) { a += ms[M0 + d]; b += ms[d * FLUX_TILE_SHAPES + best[d]]; }
        best[5] = a < b ? 1 : 0;
      }
      L->met_flux = false;
      if (P.if_viscous == 1) {
        L->met_ev = true;
        ViscArgs va = visc_args<NS>();
        va.kc = best[3];
        ms[M0 + 3] = timed([&] { visc_ev_launch<NS>(va); });
        L->met_ev = false;
        int mi = 0;
        for (int m = 0; m < 4; m++) if (VE_KC_CHOICES[m] == best[3]) mi = m;
        best[6] = ms[M0 + 3] < ms[3 * FLUX_TILE_SHAPES + mi] ? 1 : 0;
        L->met_div = true;
        DivArgs da = div_args();
        da.kc = best[4];
        ms[M0 + 4] = timed([&] { visc_div_launch(da); });
        L->met_div = false;
        int mj = 4;
        for (int m = 0; m < 4; m++) if (VE_KC_CHOICES[m] == best[4]) mj = m;
        best[7] = ms[M0 + 4] < ms[3 * FLUX_TILE_SHAPES + 4 + mj] ? 1 : 0;
      }
    }
    if (P.if_viscous == 1) {  // k_visc_ev beside the flux sweeps or after them: the whole flow
                              // right-hand side of a stage with the chosen tiles, both ways
      const int M1 = 3 * FLUX_TILE_SHAPES + 9 + 5;
      for (int d = 0; d < 3; d++) L->flux_ts[d] = best[d];
      L->kc_ev = best[3];
      L->kc_div = best[4];
      L->met_flux = best[5] && L->sep;
      L->met_ev = best[6] && L->sep;
      L->met_div = best[7] && L->sep;
      const FluxArgs fr = flow_flux_args();
      L->fork_visc = false;
      ms[M1] = timed([&] { flow_rhs_t<NS>(fr); });
      L->fork_visc = true;
      ms[M1 + 1] = timed([&] { flow_rhs_t<NS>(fr); });
      best[8] = ms[M1 + 1] < ms[M1] ? 1 : 0;
      L->fork_visc = best[8] != 0;
    }
    if (NS > 1) {  // the species chain on the third stream or in order: a stage's right-hand
                   // sides without the species RK update, both ways
      const int M2 = 3 * FLUX_TILE_SHAPES + 9 + 5 + 2;
      for (int d = 0; d < 3; d++) L->flux_ts[d] = best[d];
      L->kc_ev = best[3];
      L->kc_div = best[4];
      L->met_flux = best[5] && L->sep;
      L->met_ev = best[6] && L->sep;
      L->met_div = best[7] && L->sep;
      L->fork_visc = (best[8] & 1) != 0;
      L->fork_species = false;
      ms[M2] = timed([&] { stage_rhs_t<NS>(1, 0.0, false); });
      L->fork_species = true;
      ms[M2 + 1] = timed([&] { stage_rhs_t<NS>(1, 0.0, false); });
      best[8] = (best[8] & 1) | (ms[M2 + 1] < ms[M2] ? 2 : 0);
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  CK(cudaEventDestroy(e0));
  CK(cudaEventDestroy(e1));
}

// ---------------------------------------------------------------- filtering and analysis
// filtering (OCFD_filtering.f90:4-72) for the groups whose step interval divides istep; F is
// Para%Filter(100,10) column-major. Every pass filters the five conserved variables from an
// unfiltered copy (fn, free between steps) and leaves the primitives as they are, as the
// reference does; the shock filter first runs comput_flow_variables (krk = 0 of k_rk_prims).
template <int NS>
void filter_t(int istep, int nf, const double* F) {
  const ocfd_params& P = L->P;
  const int nn3[3] = {P.nx, P.ny, P.nz};
  const long long N = L->hc.N;
  for (int m = 0; m < nf; m++) {
    const double* c = F + 100 * m;
    if (istep % (int)std::lround(c[0]) != 0) continue;
    int b[3][2];
    for (int d = 0; d < 3; d++) {  // global -> local index of the single rank (:34-39)
      b[d][0] = std::max((int)std::lround(c[4 + 2 * d]), 1);
      b[d][1] = std::min((int)std::lround(c[5 + 2 * d]), nn3[d]);
    }
    const int scheme = (int)std::lround(c[10]);
    const double s0 = c[11], rth = c[12];
    for (int d = 0; d < 3; d++) {
      if (std::lround(c[1 + d]) != 1 || (scheme != 1 && scheme != 2)) continue;
      // the filtered direction keeps 5 (Fo9p) or 3 (shock) points off a non-periodic end
      const int edge = scheme == 1 ? 5 : 3;
      FilterBox fb;
      for (int e = 0; e < 3; e++) { fb.lo[e] = b[e][0]; fb.hi[e] = b[e][1]; }
      if (P.iperiodic[d] != 1) {
        fb.lo[d] = std::max(fb.lo[d], edge + 1);
        fb.hi[d] = std::min(fb.hi[d], nn3[d] - edge);
      }
      if (scheme == 2) prims_t<NS>(0, 0.0);  // comput_flow_variables (:208)
      const long long cells = (long long)std::max(0, fb.hi[0] - fb.lo[0] + 1) *
                              std::max(0, fb.hi[1] - fb.lo[1] + 1) * std::max(0, fb.hi[2] - fb.lo[2] + 1);
      if (cells == 0) continue;
      CK(cudaMemcpyAsync(L->fn, L->f, sizeof(double) * 5 * N, cudaMemcpyDeviceToDevice, L->st));
      KTimer t(KC_OTHER);
      const unsigned nb = nblk(cells, 256);
      if (scheme == 1) {
        if (d == 0) k_filter_fo9p<0><<<nb, 256, 0, L->st>>>(L->f, L->fn, fb, s0);
        else if (d == 1) k_filter_fo9p<1><<<nb, 256, 0, L->st>>>(L->f, L->fn, fb, s0);
        else k_filter_fo9p<2><<<nb, 256, 0, L->st>>>(L->f, L->fn, fb, s0);
      } else {
        if (d == 0) k_filter_shock<0><<<nb, 256, 0, L->st>>>(L->f, L->fn, L->p, fb, s0, rth);
        else if (d == 1) k_filter_shock<1><<<nb, 256, 0, L->st>>>(L->f, L->fn, L->p, fb, s0, rth);
        else k_filter_shock<2><<<nb, 256, 0, L->st>>>(L->f, L->fn, L->p, fb, s0, rth);
      }
      LAUNCH_CHECK();
    }
  }
}

// copy stream, events and the show_flow_msg buffers of the asynchronous save / show calls
void async_setup() {
  if (L->cst) return;
  CK(cudaStreamCreateWithFlags(&L->cst, cudaStreamNonBlocking));
  for (int m = 0; m < 2; m++) {
    CK(cudaEventCreateWithFlags(&L->snap_ready[m], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&L->snap_done[m], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&L->diag_ready, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&L->diag_done, cudaEventDisableTiming));
  CK(cudaMalloc(&L->diag_dev, sizeof(double) * 2));
  CK(cudaMallocHost(&L->diag_host, sizeof(double) * 2));
}

double* ana_partials(size_t n) {
  if (L->ana_part_n < n) {
    if (L->ana_part) CK(cudaFree(L->ana_part));
    L->ana_part = nullptr;
    CK(cudaMalloc(&L->ana_part, sizeof(double) * n));
    L->ana_part_n = n;
  }
  return L->ana_part;
}
inline double hp3(double x) { double a = x * x; return a * x; }
inline double hp4(double x) { double a = x * x; return a * a; }

double wall_ht(double tt) {
  // get_ht_multifrequancy (OCFD_BC_Boundarylayers.f90:579-618), evaluated on the host
  const double PI = 3.14159265358979;
  double beta = L->P.bc_para[13];
  if (!(beta > 0.0)) return 1.0;
  double ht = 0.0;
  for (size_t m = 0; m < L->tm.size(); m++) ht = ht + L->tm[m] * std::sin((m + 1) * beta * tt * 2.0 * PI + 2.0 * PI * L->fait[m]);
  return ht;
}

void set_time(double tt) {
  *L->ht_host = wall_ht(tt);
  CK(cudaMemcpyAsync(L->ht_dev, L->ht_host, sizeof(double), cudaMemcpyHostToDevice, L->st));
}

int check_status() {
  CK(cudaMemcpyAsync(L->shost, L->sdev, sizeof(DevStatus), cudaMemcpyDeviceToHost, L->st));
  CK(cudaStreamSynchronize(L->st));
  prof_collect();
  if (L->shost->error) {
    int e = L->shost->error;
    CK(cudaMemsetAsync(&L->sdev->error, 0, sizeof(int), L->st));
    g_err = e == OCFD_ERR_NEGATIVE_ET ? "Number of Negative Temperature Points > Limit (10)" : "device error";
    return e;
  }
  if (L->chem_mode == 1 && sg_device_error(L->st)) {
    g_err = "surrogate chemistry: a bounded wait of the network kernel ran out";
    return OCFD_ERR_TIMEOUT;
  }
  if (L->shost->chem_bad) {
    const int nb = L->shost->chem_bad;
    CK(cudaMemsetAsync(&L->sdev->chem_bad, 0, sizeof(int), L->st));
    g_err = "chemistry: " + std::to_string(nb) + " cell(s) with a zero Gauss pivot or a non-finite result";
    return OCFD_ERR_CHEM;
  }
  if (L->shost->nan_count) {
    CK(cudaMemsetAsync(&L->sdev->nan_count, 0, sizeof(int), L->st));
    g_err = "NaN in the internal energy";
    return OCFD_ERR_NAN;
  }
  return 0;
}

// outcome of a batched chemistry call from its two error words (Newton, bad reactors)
int batch_result() {
  if (L->b_last[1] > 0) {
    g_err = "chemistry: " + std::to_string(L->b_last[1]) +
            " reactor(s) with a zero Gauss pivot or a non-finite result (their values are returned as computed)";
    return OCFD_ERR_CHEM;
  }
  return 0;
}

template <class F>
int guarded(F&& fn) {
  try {
    return fn();
  } catch (CudaError& e) {
    g_err = e.what();
    return e.code;
  } catch (std::exception& e) {
    g_err = e.what();
    return OCFD_ERR_PARAM;
  }
}

void fill_thermo(DevConst& c, const ocfd_thermo* th, int realgas) {
  c.realgas = realgas;
  c.n_tct = th->n_tct;
  for (int j = 0; j < OCFD_NTCT_MAX; j++) c.tct[j] = th->tct[j];
  c.tct_max = th->tct_max;
  for (int k = 0; k < th->n_spec; k++) {
    c.Mi[k] = th->mi[k];
    c.rMi[k] = 1.0 / th->mi[k];
    c.Ri[k] = 8.314 / th->mi[k];
    double ect = 0.0;
    for (int j = 0; j < th->n_tct; j++) {
      for (int m = 0; m < 7; m++) c.cf[k][j][m] = th->coef[k][j][m];
      if (j == 0) {
        ect = 0.0;
      } else {  // read_Spec cross-range continuity offset (CHEM_thermdyn.f90:43-47)
        double t = th->tct[j - 1];
        const double* a = th->coef[k][j];
        const double* b = th->coef[k][j - 1];
        double t2 = t * t, t3 = t2 * t, t4 = t2 * t2, t5 = t2 * t3;
        double s = (a[0] - b[0]) * t + (a[1] - b[1]) * t2 / 2.0 + (a[2] - b[2]) * t3 / 3.0 +
                   (a[3] - b[3]) * t4 / 4.0 + (a[4] - b[4]) * t5 / 5.0;
        ect = -s + ect;
      }
      c.cf[k][j][7] = ect;
    }
  }
  for (int i = 0; i < th->n_spec; i++)
    for (int j = 0; j < th->n_spec; j++) c.mratio[i][j] = th->mi[i] / th->mi[j];
}
// magic pair of fast_div for a divisor d >= 1: m = ceil(2^(31 + l) / d) with l = ceil(log2 d) and
// s = l - 1, exact for every dividend below 2^31 (d = 1 is special-cased on the device); checked
// here against the hardware division on the largest dividends and a sweep of small ones
void fast_divisor(unsigned d, unsigned& m, int& s) {
  int l = 0;
  while ((1ull << l) < d) l++;
  const unsigned long long p = 1ull << (31 + l);
  m = (unsigned)((p + d - 1) / d);
  s = l > 0 ? l - 1 : 0;
  if (d <= 1) return;
  auto q = [&](unsigned n) { return (unsigned)(((unsigned long long)n * m) >> 32) >> s; };
  for (unsigned n = 0; n < 4096; n++)
    if (q(n) != n / d) throw std::runtime_error("fast_divisor");
  for (unsigned n = 0x7fffffffu; n > 0x7fffffffu - 4096; n--)
    if (q(n) != n / d) throw std::runtime_error("fast_divisor");
}

void fill_kin(DevConst& c, const ocfd_kinetics* kin) {
  c.nreac = kin->n_reac;
  c.rereac = kin->rereac;
  for (int j = 0; j < kin->n_reac; j++) {
    c.af_type[j] = kin->af_type[j];
    c.tr_reac[j] = kin->tr_reac[j];
    c.fc_troe[j] = kin->fc_troe[j];
    int sg = 0;
    (void)sg;
    for (int s = 0; s < 2; s++) { c.af[j][s] = kin->af[j][s]; c.bf[j][s] = kin->bf[j][s]; c.ef[j][s] = kin->ef[j][s]; }
    c.ar[j] = kin->ar[j]; c.br[j] = kin->br[j]; c.er[j] = kin->er[j];
    for (int m = 0; m < 5; m++) c.park[j][m] = kin->park[j][m];
    for (int i = 0; i < kin->n_spec; i++) {
      c.vf[j][i] = (signed char)kin->vf[j][i];
      c.vr[j][i] = (signed char)kin->vr[j][i];
      c.treff[j][i] = kin->treff[j][i];
      sg += kin->vr[j][i] - kin->vf[j][i];
    }
    c.sgm[j] = sg;
  }
}
void fill_trans(DevConst& c, const ocfd_transport* tr, int ns) {
  c.flag_vis = tr->flag_vis; c.flag_cond = tr->flag_cond; c.flag_diff = tr->flag_diff;
  c.amu0 = tr->amu0; c.pr = tr->pr; c.sc = tr->sc;
  for (int k = 0; k < ns; k++)
    for (int m = 0; m < 4; m++) {
      c.mu_an[k][m] = tr->mu_an[k][m];
      c.k_an[k][m] = tr->k_an[k][m];
      for (int j = 0; j < ns; j++) c.d_an[k][j][m] = tr->d_an[k][j][m];
    }
  // Wilke pair constants (needs Mi: fill_thermo runs first)
  for (int k = 0; k < ns; k++)
    for (int j = 0; j < ns; j++) {
      c.wk_a[k][j] = std::sqrt(c.Mi[j] / c.Mi[k]);
      c.wk_b[k][j] = std::sqrt(8.0 * (1.0 + c.Mi[k] / c.Mi[j]));
      c.wk_c[k][j] = std::sqrt(c.wk_a[k][j]);
      c.wk_binv[k][j] = 1.0 / c.wk_b[k][j];
    }
  int np = 0;
  for (int a = 0; a < ns; a++)
    for (int b = a + 1; b < ns; b++) {
      c.pair_a[np] = (unsigned char)a;
      c.pair_b[np] = (unsigned char)b;
      c.pair_of[a][b] = c.pair_of[b][a] = (unsigned char)np;
      np++;
    }
}

void release() {
  if (!L) return;
  if (L->gexec) cudaGraphExecDestroy(L->gexec);
  if (L->gchunk) cudaGraphExecDestroy(L->gchunk);
  if (L->gstep) cudaGraphDestroy(L->gstep);
  if (L->ht_counter) cudaFree(L->ht_counter);
  for (auto& e : L->ev_pool) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  if (L->arena) cudaFree(L->arena);
  if (L->amu_keep) cudaFree(L->amu_keep);
  if (L->met_store) cudaFree(L->met_store);
  if (L->cst) cudaStreamSynchronize(L->cst);
  for (int m = 0; m < 2; m++) {
    if (L->snap_dev[m]) cudaFree(L->snap_dev[m]);
    if (L->snap_host[m]) cudaFreeHost(L->snap_host[m]);
    if (L->snap_ready[m]) cudaEventDestroy(L->snap_ready[m]);
    if (L->snap_done[m]) cudaEventDestroy(L->snap_done[m]);
  }
  if (L->diag_dev) cudaFree(L->diag_dev);
  if (L->diag_host) cudaFreeHost(L->diag_host);
  if (L->diag_ready) cudaEventDestroy(L->diag_ready);
  if (L->diag_done) cudaEventDestroy(L->diag_done);
  if (L->cst) cudaStreamDestroy(L->cst);
  if (L->ana_part) cudaFree(L->ana_part);
  if (L->avg) cudaFree(L->avg);
  if (L->shost) cudaFreeHost(L->shost);
  if (L->ht_host) cudaFreeHost(L->ht_host);
  if (L->b_di) cudaFree(L->b_di);
  if (L->ht_seq) cudaFree(L->ht_seq);
  if (L->ht_seq_host) cudaFreeHost(L->ht_seq_host);
  for (auto& e : L->uev)
    if (e) cudaEventDestroy(e);
  if (L->ev_fork) cudaEventDestroy(L->ev_fork);
  if (L->ev_join) cudaEventDestroy(L->ev_join);
  if (L->st2) cudaStreamDestroy(L->st2);
  if (L->ev_sp_fork) cudaEventDestroy(L->ev_sp_fork);
  if (L->ev_se_done) cudaEventDestroy(L->ev_se_done);
  if (L->ev_sp_join) cudaEventDestroy(L->ev_sp_join);
  if (L->st3) cudaStreamDestroy(L->st3);
  if (L->st) cudaStreamDestroy(L->st);
  delete L;
  L = nullptr;
}

}  // namespace

// ---------------------------------------------------------------- setup kernels
namespace ocfd {
__global__ void k_fill(double* p, long long n, double v) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = v;
}
// updata_Axyz_periodic (OCFD_mesh.f90:109-185): shift the coordinates of periodic face halos
__global__ void k_shift(double* X, double* Y, double* Z, int dir, double sx, double sy, double sz) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int L = OCFD_L;
  int a, b, l, side;
  long long na = dir == 0 ? cC.ny : cC.nx, nb = dir == 2 ? cC.ny : cC.nz;
  if (t >= 2 * L * na * nb) return;
  side = (int)(t & 1);
  long long r = t >> 1;
  a = (int)(r % na) + 1;
  l = (int)((r / na) % L);
  b = (int)(r / na / L) + 1;
  int n = dir == 0 ? cC.nx : (dir == 1 ? cC.ny : cC.nz);
  int s = side == 0 ? 1 - L + l : n + 1 + l;
  int q = dir == 0 ? hidx(s, a, b) : (dir == 1 ? hidx(a, s, b) : hidx(a, b, s));
  if (side == 0) { X[q] = X[q] - sx; Y[q] = Y[q] - sy; Z[q] = Z[q] - sz; }
  else { X[q] = X[q] + sx; Y[q] = Y[q] + sy; Z[q] = Z[q] + sz; }
}
// comput_Jacobian3d (OCFD_mesh.f90:60-107) for general grids
__global__ void k_jacobian(const double* X, const double* Y, const double* Z, double* const* m) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  int q = hidx(i, j, k);
  double xi1 = cdiff(X, q, 0, i, cC.nx), yi1 = cdiff(Y, q, 0, i, cC.nx), zi1 = cdiff(Z, q, 0, i, cC.nx);
  double xj1 = cdiff(X, q, 1, j, cC.ny), yj1 = cdiff(Y, q, 1, j, cC.ny), zj1 = cdiff(Z, q, 1, j, cC.ny);
  double xk1 = cdiff(X, q, 2, k, cC.nz), yk1 = cdiff(Y, q, 2, k, cC.nz), zk1 = cdiff(Z, q, 2, k, cC.nz);
  double jac = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 - yi1 * xj1 * zk1 -
                      xi1 * zj1 * yk1);
  m[G_AJAC][q] = jac;
  m[G_AKX][q] = jac * (yj1 * zk1 - zj1 * yk1);
  m[G_AKY][q] = jac * (zj1 * xk1 - xj1 * zk1);
  m[G_AKZ][q] = jac * (xj1 * yk1 - yj1 * xk1);
  m[G_AIX][q] = jac * (yk1 * zi1 - zk1 * yi1);
  m[G_AIY][q] = jac * (zk1 * xi1 - xk1 * zi1);
  m[G_AIZ][q] = jac * (xk1 * yi1 - yk1 * xi1);
  m[G_ASX][q] = jac * (yi1 * zj1 - zi1 * yj1);
  m[G_ASY][q] = jac * (zi1 * xj1 - xi1 * zj1);
  m[G_ASZ][q] = jac * (xi1 * yj1 - yi1 * xj1);
}
// Akx1 = Akx / Ajac ... over the full halo range (OCFD_mesh.f90:40-54)
__global__ void k_metric_ratio(double* const* m, long long H) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= H) return;
  double jac = m[G_AJAC][t];
  for (int a = 0; a < 9; a++) m[G_AKX1 + a][t] = m[a][t] / jac;
}
// Jac_Ghost_Boundary (OCFD_GhostCell.f90:1-160, 366-580) on the ghost slab of one face: LAP planes
// outside the face, tangential interior range. Thread t -> (depth 1..LAP, tangential a, b).
__device__ __forceinline__ bool ghost_point(int face, long long t, int& g, int& a, int& b, int& n) {
  const int dir = face / 2, side = face % 2;
  n = dir == 0 ? cC.nx : (dir == 1 ? cC.ny : cC.nz);
  const int ta = dir == 0 ? cC.ny : cC.nx, tb = dir == 2 ? cC.ny : cC.nz;
  if (t >= (long long)ta * tb * OCFD_L) return false;
  a = (int)(t % ta) + 1;
  const int l = (int)((t / ta) % OCFD_L) + 1;
  b = (int)(t / ta / OCFD_L) + 1;
  g = side == 0 ? 1 - l : n + l;
  return true;
}
__device__ __forceinline__ int face_at(int dir, int s, int a, int b) {
  return dir == 0 ? hidx(s, a, b) : (dir == 1 ? hidx(a, s, b) : hidx(a, b, s));
}
// Ghost_Cell = 1: copy the face plane's metrics, extrapolate the coordinates linearly
__global__ void k_jac_ghost1(int face, double* X, double* Y, double* Z, double* const* m) {
  int g, a, b, n;
  if (!ghost_point(face, (long long)blockIdx.x * blockDim.x + threadIdx.x, g, a, b, n)) return;
  const int dir = face / 2, side = face % 2;
  const int qg = face_at(dir, g, a, b), qb = face_at(dir, side == 0 ? 1 : n, a, b);
  const int q2 = face_at(dir, side == 0 ? 2 : n - 1, a, b);
  for (int k = 0; k < 10; k++) m[k][qg] = m[k][qb];
  const double f = side == 0 ? (1.0 - g) : (double)(g - n);
  X[qg] = X[qb] + f * (X[qb] - X[q2]);
  Y[qg] = Y[qb] + f * (Y[qb] - Y[q2]);
  Z[qg] = Z[qb] + f * (Z[qb] - Z[q2]);
}
// Ghost_Cell = 2: mirror the coordinates (x_g = 2 x_b - x_mirror) ...
__global__ void k_jac_ghost2_coords(int face, double* X, double* Y, double* Z) {
  int g, a, b, n;
  if (!ghost_point(face, (long long)blockIdx.x * blockDim.x + threadIdx.x, g, a, b, n)) return;
  const int dir = face / 2, side = face % 2;
  const int qg = face_at(dir, g, a, b), qb = face_at(dir, side == 0 ? 1 : n, a, b);
  const int qm = face_at(dir, side == 0 ? 2 - g : 2 * n - g, a, b);
  X[qg] = 2.0 * X[qb] - X[qm];
  Y[qg] = 2.0 * Y[qb] - Y[qm];
  Z[qg] = 2.0 * Z[qb] - Z[qm];
}
// ... and recompute the metrics there (comput_Jacobian3d_Ghost): derivatives one-sided at the ends
// of each range, 2nd-order central next to them, 4th-order central elsewhere
__global__ void k_jac_ghost2_metric(int face, const double* X, const double* Y, const double* Z, double* const* m) {
  int g, a, b, n;
  if (!ghost_point(face, (long long)blockIdx.x * blockDim.x + threadIdx.x, g, a, b, n)) return;
  const int dir = face / 2, side = face % 2;
  int lo[3] = {1, 1, 1}, hi[3] = {cC.nx, cC.ny, cC.nz};
  lo[dir] = side == 0 ? 1 - OCFD_L : n;
  hi[dir] = side == 0 ? 1 : n + OCFD_L;
  int i = dir == 0 ? g : a, j = dir == 0 ? a : (dir == 1 ? g : b), k = dir == 2 ? g : b;
  if (dir == 2) { i = a; j = b; }
  const int q = hidx(i, j, k);
  const int pos[3] = {i, j, k};
  auto der = [&](const double* A, int dd) {
    const double* f = A + q;
    const int s = hstride(dd);
    const double h = cC.h[dd];
    const int ps = pos[dd];
    if (ps == lo[dd]) return (-3.0 * f[0] + 4.0 * f[s] - f[2 * s]) / (2.0 * h);
    if (ps == hi[dd]) return (f[-2 * s] - 4.0 * f[-s] + 3.0 * f[0]) / (2.0 * h);
    if (ps == lo[dd] + 1 || ps == hi[dd] - 1) return (f[s] - f[-s]) / (2.0 * h);
    return (8.0 * (f[s] - f[-s]) - (f[2 * s] - f[-2 * s])) / (12.0 * h);
  };
  double xi1 = der(X, 0), yi1 = der(Y, 0), zi1 = der(Z, 0);
  double xj1 = der(X, 1), yj1 = der(Y, 1), zj1 = der(Z, 1);
  double xk1 = der(X, 2), yk1 = der(Y, 2), zk1 = der(Z, 2);
  double jac = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 - yi1 * xj1 * zk1 -
                      xi1 * zj1 * yk1);
  m[G_AJAC][q] = jac;
  m[G_AKX][q] = jac * (yj1 * zk1 - zj1 * yk1);
  m[G_AKY][q] = jac * (zj1 * xk1 - xj1 * zk1);
  m[G_AKZ][q] = jac * (xj1 * yk1 - yj1 * xk1);
  m[G_AIX][q] = jac * (yk1 * zi1 - zk1 * yi1);
  m[G_AIY][q] = jac * (zk1 * xi1 - xk1 * zi1);
  m[G_AIZ][q] = jac * (xk1 * yi1 - yk1 * xi1);
  m[G_ASX][q] = jac * (yi1 * zj1 - zi1 * yj1);
  m[G_ASY][q] = jac * (zi1 * xj1 - xi1 * zj1);
  m[G_ASZ][q] = jac * (xi1 * yj1 - yi1 * xj1);
}
// tensor-product grids: dx/dxi(i), dy/deta(j), dz/dzeta(k) with the same CD6/CD8 + closures
__global__ void k_metric1d(const double* X, const double* Y, const double* Z, double* dx, double* dy, double* dz) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int L = OCFD_L;
  if (t < cC.nx) dx[t + L] = cdiff(X, hidx(t + 1, 1, 1), 0, t + 1, cC.nx);
  if (t < cC.ny) dy[t + L] = cdiff(Y, hidx(1, t + 1, 1), 1, t + 1, cC.ny);
  if (t < cC.nz) dz[t + L] = cdiff(Z, hidx(1, 1, t + 1), 2, t + 1, cC.nz);
}
__global__ void k_metric1d_halo(double* dx, double* dy, double* dz) {
  int l = threadIdx.x;
  const int L = OCFD_L;
  if (l >= L) return;
  double* a[3] = {dx, dy, dz};
  int n[3] = {cC.nx, cC.ny, cC.nz};
  for (int dd = 0; dd < 3; dd++) {
    if (cC.iper[dd]) {
      a[dd][l] = a[dd][n[dd] + l];          // index s+L-1 for s = 1-L+l  <-  s = n-L+1+l
      a[dd][n[dd] + L + l] = a[dd][L + l];  // s = n+1+l  <-  s = 1+l
    } else {
      a[dd][l] = 1.0;
      a[dd][n[dd] + L + l] = 1.0;
    }
  }
}
// cross derivatives of the coordinates on the non-periodic end planes (closure residues)
__global__ void k_metric_edges(const double* X, const double* Y, const double* Z, double* const* e) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int L = OCFD_L, nx = cC.nx, ny = cC.ny, nz = cC.nz;
  for (int s = 0; s < 2; s++) {
    int is = s ? nx : 1, js = s ? ny : 1, ks = s ? nz : 1;
    if (t < ny) e[E_YI][s * (ny + 2 * L) + t + L] = cdiff(Y, hidx(is, t + 1, 1), 0, is, nx);
    if (t < nz) e[E_ZI][s * (nz + 2 * L) + t + L] = cdiff(Z, hidx(is, 1, t + 1), 0, is, nx);
    if (t < nx) e[E_XJ][s * (nx + 2 * L) + t + L] = cdiff(X, hidx(t + 1, js, 1), 1, js, ny);
    if (t < nz) e[E_ZJ][s * (nz + 2 * L) + t + L] = cdiff(Z, hidx(1, js, t + 1), 1, js, ny);
    if (t < nx) e[E_XK][s * (nx + 2 * L) + t + L] = cdiff(X, hidx(t + 1, 1, ks), 2, ks, nz);
    if (t < ny) e[E_YK][s * (ny + 2 * L) + t + L] = cdiff(Y, hidx(1, t + 1, ks), 2, ks, nz);
  }
}
__global__ void k_metric_edges_halo(double* const* e) {
  int l = threadIdx.x;
  const int L = OCFD_L;
  if (l >= L) return;
  const int dir[6] = {1, 2, 0, 2, 0, 1};  // the index direction of each end-plane array
  const int n[3] = {cC.nx, cC.ny, cC.nz};
  for (int m = 0; m < 6; m++)
    for (int s = 0; s < 2; s++) {
      int d = dir[m], nn = n[d];
      double* a = e[m] + s * (nn + 2 * L);
      if (cC.iper[d]) {
        a[l] = a[nn + l];
        a[nn + L + l] = a[L + l];
      } else {
        a[l] = 0.0;
        a[nn + L + l] = 0.0;
      }
    }
}
// the ten reference metric arrays from the separable representation (for downloads); halo
// points the reference never fills keep allocate_flow_data's 1.0
__global__ void k_expand_metrics(Geo g, double* out, long long H) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= H) return;
  int i = (int)(t % cC.HX) - OCFD_L + 1;
  int j = (int)((t / cC.HX) % cC.HY) - OCFD_L + 1;
  int k = (int)(t / cC.HX / cC.HY) - OCFD_L + 1;
  if (metric_unfilled(i, j, k)) {
    for (int m = 0; m < 10; m++) out[m * H + t] = 1.0;
    return;
  }
  double a[9], a1[9];
  metric_all<true>(g, i, j, k, (int)t, a, a1);
  for (int m = 0; m < 9; m++) out[m * H + t] = a[m];
  out[9 * H + t] = metric_jac<true>(g, i, j, k, (int)t);
}
// FP64 FMA throughput probe: eight independent chains per thread, registers only
__global__ void k_fp64_peak(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int it = 0; it < iters; it++) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 1234.5678) out[0] = s;  // keeps the chains live
}
}  // namespace ocfd

namespace ocfd {
// the species count and the stream of the current set-up (ocfd_gpu_init or ocfd_gpu_chem_setup),
// for the surrogate module
int current_nspec() { return L && L->have_kin ? L->NS : 0; }
int current_const_p() { return L && L->have_kin ? L->hc.const_p : 0; }
int current_mech() { return L && L->have_kin && L->mech_on ? mech_match(L->hc) : 0; }
int current_timeadv() { return L ? L->hc.timeadv : 0; }
cudaStream_t current_stream() { return L ? L->st : nullptr; }
}  // namespace ocfd

namespace {

int validate(const ocfd_params* p) {
  auto bad = [](const char* m) { g_err = m; return OCFD_ERR_PARAM; };
  if (p->lap != 4) return bad("LAP must be 4");
  if (p->nx < 8 || p->ny < 8 || p->nz < 8) return bad("nx, ny, nz must be >= 8");
  if (p->n_spec < 1 || p->n_spec > 9) return bad("N_SPEC must be 1..9");
  int s = p->scheme_invis;
  if (!(s == 1 || s == 2 || s == 3 || s == 4 || s == 10)) return bad("Scheme_Invis must be WENO5/WENO7/OMP6/UD7L/HYBRID");
  if (!(p->scheme_vis == OCFD_SCHEME_CD6 || p->scheme_vis == OCFD_SCHEME_CD8)) return bad("Scheme_Vis must be CD6 or CD8");
  if (!(p->flux_splitting == 1 || p->flux_splitting == 2)) return bad("Flux_Splitting must be 1 or 2");
  for (int m = 0; m < 6; m++) {
    if (p->scheme_boundary[m] < -1 || p->scheme_boundary[m] > 1) return bad("Scheme_boundary must be -1, 0 or 1");
    if (p->ghost_cell[m] < 0 || p->ghost_cell[m] > 2) {
      // Ghost_Cell = -1 is the reference's user-defined ghost cell (OCFD_GhostCell_UserDef.f90)
      g_err = "Ghost_Cell must be 0, 1 or 2 (user-defined ghost cells are not carried)";
      return OCFD_ERR_UNSUPPORTED;
    }
  }
  if (p->if_scheme_character != 0 && p->if_scheme_character != 1) { g_err = "IF_Scheme_Character must be 0 or 1"; return OCFD_ERR_PARAM; }
  if (!(p->ibc == OCFD_BC_NONE || p->ibc == OCFD_BC_BOUNDARYLAYER || p->ibc == OCFD_BC_JET)) { g_err = "boundary condition not built (BC_NONE, BC_BOUNDARYLAYER, BC_JET)"; return OCFD_ERR_UNSUPPORTED; }
  if (p->wall_catalysis != 0) return bad("only non-catalytic walls");
  if (!(p->chem_timeadv == 1 || p->chem_timeadv == 2 || p->chem_timeadv == 3 || p->chem_timeadv == -1)) return bad("CHEM_TimeAdv must be 1, 2, 3 or -1");
  return 0;
}

bool separable(const ocfd_params* p, const double* coords) {
  const int L4 = OCFD_L;
  long long HX = p->nx + 2 * L4, HY = p->ny + 2 * L4;
  auto ih = [&](int i, int j, int k) { return (long long)(i + L4 - 1) + HX * ((j + L4 - 1) + HY * (long long)(k + L4 - 1)); };
  long long H = HX * HY * (p->nz + 2 * L4);
  const double* X = coords;
  const double* Y = coords + H;
  const double* Z = coords + 2 * H;
  for (int k = 1; k <= p->nz; k++)
    for (int j = 1; j <= p->ny; j++)
      for (int i = 1; i <= p->nx; i++) {
        long long q = ih(i, j, k);
        if (X[q] != X[ih(i, 1, 1)] || Y[q] != Y[ih(1, j, 1)] || Z[q] != Z[ih(1, 1, k)]) return false;
      }
  // the periodic shifts must keep the cross coordinates constant too
  for (int dd = 0; dd < 3; dd++)
    if (p->iperiodic[dd])
      for (int c = 0; c < 3; c++)
        if (c != dd && p->periodic_span[dd][c] != 0.0) return false;
  return true;
}

void set_geo_device_ptrs() {
  Geo& g = L->geo;
  for (int m = 0; m < 19; m++) g.m[m] = L->met[m];
  for (int m = 0; m < 3; m++) g.d1[m] = L->d1[m];
  for (int m = 0; m < 6; m++) g.e[m] = L->edge[m];
}

}  // namespace

extern "C" {

int ocfd_gpu_init(const ocfd_params* p, const ocfd_thermo* th, const ocfd_kinetics* kin, const ocfd_transport* tr,
                  const ocfd_bcdata* bc, const double* coords, const double* metrics) {
  return guarded([&]() -> int {
    release();
    if (!p || !th || !tr || !coords) { g_err = "null argument"; return OCFD_ERR_PARAM; }
    int e = validate(p);
    if (e) return e;
    if (th->n_spec != p->n_spec) { g_err = "thermo n_spec differs from N_SPEC"; return OCFD_ERR_PARAM; }
    if ((p->ibc == OCFD_BC_BOUNDARYLAYER || p->ibc == OCFD_BC_JET) && !bc) { g_err = "BC_BOUNDARYLAYER / BC_JET need boundary data"; return OCFD_ERR_PARAM; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { g_err = "no CUDA device"; return OCFD_ERR_CUDA; }
    L = new Lib();
    L->P = *p;
    L->NS = p->n_spec;
    CK(cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&L->st2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&L->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&L->ev_join, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&L->st3, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&L->ev_sp_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&L->ev_se_done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&L->ev_sp_join, cudaEventDisableTiming));
    DevConst& c = L->hc;
    c.nx = p->nx; c.ny = p->ny; c.nz = p->nz; c.ns = p->n_spec;
    fast_divisor((unsigned)p->nx, c.mx, c.sx);
    fast_divisor((unsigned)p->ny, c.my, c.sy);
    c.jt = 1;
    while (c.jt < 32 && p->ny % (2 * c.jt) == 0) c.jt *= 2;
    fast_divisor((unsigned)(c.jt * p->nx), c.m_slab, c.s_slab);
    fast_divisor((unsigned)(c.jt * p->nx * p->nz), c.m_tile, c.s_tile);
    c.HX = p->nx + 2 * OCFD_L; c.HY = p->ny + 2 * OCFD_L; c.HZ = p->nz + 2 * OCFD_L;
    c.H = (long long)c.HX * c.HY * c.HZ;
    c.N = (long long)p->nx * p->ny * p->nz;
    if (c.H * p->n_spec >= (1LL << 31)) { g_err = "grid too large for 32-bit halo indexing"; return OCFD_ERR_PARAM; }
    int nn[3] = {p->nx, p->ny, p->nz};
    for (int dd = 0; dd < 3; dd++) {
      c.iper[dd] = p->iperiodic[dd];
      c.bound[dd][0] = c.bound[dd][1] = p->iperiodic[dd] == 0 ? 1 : 0;
      double h = 1.0 / (nn[dd] - 1.0);
      c.h[dd] = h;
      c.h1[dd] = 1.0 / h;
      c.cd6[dd][0] = 1.0 / (60.0 * h); c.cd6[dd][1] = -3.0 / (20.0 * h); c.cd6[dd][2] = 3.0 / (4.0 * h);
      c.cd8[dd][0] = 0.8 / h; c.cd8[dd][1] = -0.2 / h; c.cd8[dd][2] = 3.80952380952380952e-2 / h;
      c.cd8[dd][3] = -3.571428571428571428e-3 / h;
      c.h2x[dd] = 2.0 * h; c.h12x[dd] = 12.0 * h;
    }
    for (int m = 0; m < 6; m++) { c.sb[m] = p->scheme_boundary[m]; c.ghost[m] = p->ghost_cell[m]; }
    c.scheme = p->scheme_invis; c.split = p->flux_splitting;
    switch (c.scheme) {
      case 1: c.Ka1 = -2; c.Kb1 = 2; c.Ka2 = -1; c.Kb2 = 3; break;
      case 2: c.Ka1 = -3; c.Kb1 = 3; c.Ka2 = -2; c.Kb2 = 4; break;
      default: c.Ka1 = -3; c.Kb1 = 4; c.Ka2 = -3; c.Kb2 = 4;
    }
    {
      const double UD7[8] = {-3.0, 25.0, -101.0, 319.0, 214.0, -38.0, 4.0, 0.0};
      const double CD8[8] = {-3.0, 29.0, -139.0, 533.0, 533.0, -139.0, 29.0, -3.0};
      for (int k = 0; k < 8; k++) c.UD7L[k] = p->ud7l_diss * UD7[k] / 420.0 + (1.0 - p->ud7l_diss) * CD8[k] / 840.0;
    }
    c.theta1 = p->hybrid_para[1];
    c.theta2 = p->hybrid_para[2];
    c.cd8_on = p->scheme_vis == OCFD_SCHEME_CD8;
    c.if_viscous = p->if_viscous;
    c.if_mass_force = p->if_mass_force;
    for (int m = 0; m < 3; m++) c.mass_force[m] = p->mass_force[m];
    fill_thermo(c, th, p->if_realgas);
    fill_trans(c, tr, p->n_spec);
    c.timeadv = p->chem_timeadv;
    if (kin) {
      if (kin->n_spec != p->n_spec || kin->n_reac > OCFD_MAX_REAC) { g_err = "kinetics size"; return OCFD_ERR_PARAM; }
      fill_kin(c, kin);
      L->have_kin = true;
    }
    CK(cudaMemcpyToSymbol(cC, &c, sizeof(DevConst)));

    L->sep = metrics == nullptr && separable(p, coords);  // given metrics are used as given
    for (int m = 0; m < 6; m++)
      if (p->ghost_cell[m] != 0) L->sep = false;  // ghost slabs carry their own metrics
    const long long H = c.H, N = c.N;
    const int NS = p->n_spec;
    size_t total = 0;
    auto add = [&](size_t n, size_t sz) { total += (n * sz + 255) & ~(size_t)255; };
    add(5 * N, 8); add(5 * N, 8); add(5 * N, 8);
    for (int m = 0; m < 8; m++) add(H, 8);
    add(NS * H, 8); add(NS * N, 8); add(H, 8);
    for (int m = 0; m < 12; m++) add(H, 8);
    if (NS > 1) {
      add(N, 8); add(N, 8); add(NS * N, 8);                              // amu, amk, amd
      for (int m = 0; m < 3; m++) add(N, 8);                             // qp
      add(NS * H, 8); for (int m = 0; m < 3; m++) add(NS * H, 8);        // ci, se
      add(NS * N, 8);                                                    // dus
    }
    for (int m = 0; m < 3; m++) add(H, 8);
    if (!L->sep) for (int m = 0; m < 19; m++) add(H, 8);
    for (int m = 0; m < 3; m++) add(nn[m] + 2 * OCFD_L, 8);
    for (int m = 0; m < 6; m++) add(2 * (std::max(nn[0], std::max(nn[1], nn[2])) + 2 * OCFD_L), 8);
    add(6, sizeof(double*));
    add(2 * ((N + 255) / 256) + 2, 8);
    size_t nv = 5 + NS;
    add(nv * (size_t)std::max((long long)p->ny * p->nz, (long long)p->nx * p->nz) + nv, 8);
    add(nv * (size_t)std::max((long long)p->ny * p->nz, (long long)p->nx * p->nz) + nv, 8);
    add((size_t)p->nx * p->nz, 8); add((size_t)p->nx * p->nz, 4); add(1, 8);
    add(6 * 20, 4); add(1, sizeof(DevStatus)); add(12, sizeof(double*)); add(19, sizeof(double*));
    L->arena_size = total + (1 << 20);
    CK(cudaMalloc(&L->arena, L->arena_size));
    CK(cudaMallocHost(&L->shost, sizeof(DevStatus)));
    CK(cudaMallocHost(&L->ht_host, sizeof(double)));

    L->f = alloc<double>(5 * N); L->fn = alloc<double>(5 * N); L->du = alloc<double>(5 * N);
    L->d = alloc<double>(H); L->u = alloc<double>(H); L->v = alloc<double>(H); L->w = alloc<double>(H);
    L->T = alloc<double>(H); L->p = alloc<double>(H); L->Et[0] = alloc<double>(H); L->Et[1] = alloc<double>(H);
    L->di = alloc<double>(NS * H); L->din = alloc<double>(NS * N); L->Rh = alloc<double>(H);
    for (int m = 0; m < 12; m++) L->ev[m] = alloc<double>(H);
    if (NS > 1) {
      L->amu = alloc<double>(N); L->amk = alloc<double>(N); L->amd = alloc<double>(NS * N);
      for (int m = 0; m < 3; m++) L->qp[m] = alloc<double>(N);
      L->ci = alloc<double>((size_t)NS * H);
      for (int m = 0; m < 3; m++) L->se[m] = alloc<double>((size_t)NS * H);
      L->dus = alloc<double>((size_t)NS * N);
    }
    L->X = alloc<double>(H); L->Y = alloc<double>(H); L->Z = alloc<double>(H);
    if (!L->sep) for (int m = 0; m < 19; m++) L->met[m] = alloc<double>(H);
    for (int m = 0; m < 3; m++) L->d1[m] = alloc<double>(nn[m] + 2 * OCFD_L);
    const int emax = std::max(nn[0], std::max(nn[1], nn[2])) + 2 * OCFD_L;
    for (int m = 0; m < 6; m++) L->edge[m] = alloc<double>(2 * emax);
    double** edge_ptrs = alloc<double*>(6);
    L->partial = alloc<double>(2 * ((N + 255) / 256) + 2);
    L->inlet = alloc<double>(nv * (size_t)std::max((long long)p->ny * p->nz, (long long)p->nx * p->nz) + nv);
    L->upper = alloc<double>(nv * (size_t)std::max((long long)p->ny * p->nz, (long long)p->nx * p->nz) + nv);
    L->wall = alloc<double>((size_t)p->nx * p->nz);
    L->nonref = alloc<int>((size_t)p->nx * p->nz);
    L->ht_dev = alloc<double>(1);
    L->patches = alloc<int>(6 * 20);
    L->sdev = alloc<DevStatus>(1);
    double** met_ptrs = alloc<double*>(19);
    CK(cudaMemsetAsync(L->sdev, 0, sizeof(DevStatus), L->st));

    // allocate_flow_data initial values (OCFD_allocate_data.f90:53-67)
    auto fill = [&](double* a, long long n, double val) {
      k_fill<<<nblk(n, 256), 256, 0, L->st>>>(a, n, val);
      LAUNCH_CHECK();
    };
    fill(L->du, 5 * N, 0.0);
    fill(L->f, 5 * N, 0.0); fill(L->fn, 5 * N, 0.0);
    for (double* a : {L->d, L->u, L->v, L->w, L->p, L->Et[0], L->Et[1]}) fill(a, H, 1.0);
    fill(L->T, H, 300.0);
    fill(L->di, NS * H, 1.0); fill(L->din, NS * N, 1.0);
    fill(L->Rh, H, 0.0);
    for (int m = 0; m < 12; m++) fill(L->ev[m], H, 0.0);
    if (NS > 1) {
      fill(L->amu, N, 0.0); fill(L->amk, N, 0.0); fill(L->amd, NS * N, 0.0);
      for (int m = 0; m < 3; m++) fill(L->qp[m], N, 0.0);
      fill(L->ci, (size_t)NS * H, 0.0);
      for (int m = 0; m < 3; m++) fill(L->se[m], (size_t)NS * H, 0.0);
      fill(L->dus, (size_t)NS * N, 0.0);
    }
    // init_mesh
    CK(cudaMemcpyAsync(L->X, coords, sizeof(double) * H, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(L->Y, coords + H, sizeof(double) * H, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(L->Z, coords + 2 * H, sizeof(double) * H, cudaMemcpyHostToDevice, L->st));
    exchange({L->X, L->Y, L->Z}, 7);
    for (int dd = 0; dd < 3; dd++) {
      if (!p->iperiodic[dd]) continue;
      long long na = dd == 0 ? p->ny : p->nx, nb = dd == 2 ? p->ny : p->nz;
      k_shift<<<nblk(2 * OCFD_L * na * nb, 256), 256, 0, L->st>>>(L->X, L->Y, L->Z, dd, p->periodic_span[dd][0],
                                                                  p->periodic_span[dd][1], p->periodic_span[dd][2]);
      LAUNCH_CHECK();
    }
    if (L->sep && metrics == nullptr) {
      int mx = std::max(p->nx, std::max(p->ny, p->nz));
      k_metric1d<<<nblk(mx, 128), 128, 0, L->st>>>(L->X, L->Y, L->Z, L->d1[0], L->d1[1], L->d1[2]);
      LAUNCH_CHECK();
      k_metric1d_halo<<<1, 32, 0, L->st>>>(L->d1[0], L->d1[1], L->d1[2]);
      LAUNCH_CHECK();
      CK(cudaMemcpyAsync(edge_ptrs, L->edge, sizeof(double*) * 6, cudaMemcpyHostToDevice, L->st));
      k_metric_edges<<<nblk(mx, 128), 128, 0, L->st>>>(L->X, L->Y, L->Z, edge_ptrs);
      LAUNCH_CHECK();
      k_metric_edges_halo<<<1, 32, 0, L->st>>>(edge_ptrs);
      LAUNCH_CHECK();
    } else {
      L->sep = false;
      if (!L->met[0]) throw std::runtime_error("metric arrays not allocated");
      CK(cudaMemcpyAsync(met_ptrs, L->met, sizeof(double*) * 19, cudaMemcpyHostToDevice, L->st));
      for (int m = 0; m < 19; m++) fill(L->met[m], H, 1.0);
      if (metrics) {
        for (int m = 0; m < 10; m++)
          CK(cudaMemcpyAsync(L->met[m], metrics + (size_t)m * H, sizeof(double) * H, cudaMemcpyHostToDevice, L->st));
      } else {
        k_jacobian<<<nblk(N, 256), 256, 0, L->st>>>(L->X, L->Y, L->Z, met_ptrs);
        LAUNCH_CHECK();
      }
      std::vector<double*> ml(L->met, L->met + 10);
      exchange_v(ml, 7);
      // Jac_Ghost_boundary: all Ghost_Cell = 1 faces, then the Ghost_Cell = 2 faces
      for (int pass = 1; pass <= 2; pass++)
        for (int face = 0; face < 6; face++) {
          if (p->ghost_cell[face] != pass) continue;
          const int dir = face / 2;
          const long long na = dir == 0 ? p->ny : p->nx, nb = dir == 2 ? p->ny : p->nz;
          const unsigned nbk = nblk(na * nb * OCFD_L, 128);
          if (pass == 1) {
            k_jac_ghost1<<<nbk, 128, 0, L->st>>>(face, L->X, L->Y, L->Z, met_ptrs);
          } else {
            k_jac_ghost2_coords<<<nbk, 128, 0, L->st>>>(face, L->X, L->Y, L->Z);
            k_jac_ghost2_metric<<<nbk, 128, 0, L->st>>>(face, L->X, L->Y, L->Z, met_ptrs);
          }
          LAUNCH_CHECK();
        }
      k_metric_ratio<<<nblk(H, 256), 256, 0, L->st>>>(met_ptrs, H);
      LAUNCH_CHECK();
    }
    set_geo_device_ptrs();

    // boundary-layer data (init_bcdata_boundary / init_bc_nonRef / init_bc_wall_perturbation)
    if (p->ibc == OCFD_BC_BOUNDARYLAYER) {
      L->inlet_kind = (int)std::lround(p->bc_para[0]);
      L->upper_kind = (int)std::lround(p->bc_para[1]);
      L->outlet = (int)std::lround(p->bc_para[3]);
      size_t ni = L->inlet_kind == 0 ? nv : (L->inlet_kind == 1 ? nv * p->ny : nv * (size_t)p->ny * p->nz);
      size_t nu = L->upper_kind == 0 ? nv : (L->upper_kind == 1 ? nv * p->nx : nv * (size_t)p->nx * p->nz);
      if (L->inlet_kind < 0 || L->inlet_kind > 2 || L->upper_kind > 2) { g_err = "BcData_inlet / BcData_upper"; return OCFD_ERR_PARAM; }
      CK(cudaMemcpyAsync(L->inlet, bc->inlet, sizeof(double) * ni, cudaMemcpyHostToDevice, L->st));
      if (L->upper_kind >= 0) CK(cudaMemcpyAsync(L->upper, bc->upper, sizeof(double) * nu, cudaMemcpyHostToDevice, L->st));
      if (bc->wall_pertb) CK(cudaMemcpyAsync(L->wall, bc->wall_pertb, sizeof(double) * p->nx * p->nz, cudaMemcpyHostToDevice, L->st));
      else fill(L->wall, (long long)p->nx * p->nz, 0.0);
      L->tm.assign(bc->tm, bc->tm + bc->n_tm);
      L->fait.assign(bc->fait, bc->fait + bc->n_tm);
      std::vector<int> nr((size_t)p->nx * p->nz, 0);
      int mode = (int)std::lround(p->bc_para[2]);
      double sy0 = std::tan(p->aoa);
      const int L4 = OCFD_L;
      long long HX = c.HX, HY = c.HY;
      auto ih = [&](int i, int j, int k) { return (long long)(i + L4 - 1) + HX * ((j + L4 - 1) + HY * (long long)(k + L4 - 1)); };
      const double* Xh = coords;
      const double* Yh = coords + H;
      for (int k = 1; k <= p->nz; k++)
        for (int i = 1; i <= p->nx; i++) {
          int val = 0;
          if (mode == 1) val = 1;
          else if (mode == 0) {
            double sy;
            if (i == 1) sy = (Yh[ih(i + 1, p->ny, k)] - Yh[ih(i, p->ny, k)]) / (Xh[ih(i + 1, p->ny, k)] - Xh[ih(i, p->ny, k)]);
            else sy = (Yh[ih(i, p->ny, k)] - Yh[ih(i - 1, p->ny, k)]) / (Xh[ih(i, p->ny, k)] - Xh[ih(i - 1, p->ny, k)]);
            val = (sy >= sy0 + 1.0e-6) ? 0 : 1;
          }
          nr[(i - 1) + (size_t)p->nx * (k - 1)] = val;
        }
      CK(cudaMemcpy(L->nonref, nr.data(), sizeof(int) * nr.size(), cudaMemcpyHostToDevice));
    }
    if (p->ibc == OCFD_BC_JET) {  // ocfd_bc_jet: BcData_inlet = 2, no upper data
      L->inlet_kind = 2;
      L->upper_kind = -1;
      CK(cudaMemcpyAsync(L->inlet, bc->inlet, sizeof(double) * nv * p->ny * p->nz, cudaMemcpyHostToDevice, L->st));
    }
    // hybrid forced patches (Hybrid_para(4..), OCFD_SetHybrid.f90:80-102)
    if (p->scheme_invis == OCFD_SCHEME_HYBRID) {
      int mp = (int)std::lround(p->hybrid_para[3]);
      if (mp < 0 || mp > 15) { g_err = "Hybrid_para(4): at most 15 patches"; return OCFD_ERR_PARAM; }
      std::vector<int> pb(6 * 20, 0);
      for (int m = 0; m < mp; m++) {
        const double* h = p->hybrid_para + 4 + 6 * m;
        pb[6 * m + 0] = std::max((int)std::lround(h[0]), 1);
        pb[6 * m + 1] = std::min((int)std::lround(h[1]), p->nx);
        pb[6 * m + 2] = std::max((int)std::lround(h[2]), 1);
        pb[6 * m + 3] = std::min((int)std::lround(h[3]), p->ny);
        pb[6 * m + 4] = std::max((int)std::lround(h[4]), 1);
        pb[6 * m + 5] = std::min((int)std::lround(h[5]), p->nz);
      }
      L->npatch = mp;
      CK(cudaMemcpy(L->patches, pb.data(), sizeof(int) * pb.size(), cudaMemcpyHostToDevice));
    }
    CK(cudaStreamSynchronize(L->st));
    return 0;
  });
}

int ocfd_gpu_init_state(const double* prim5, const double* di, double tt) {
  return guarded([&]() -> int {
    if (!L || !L->d) { g_err = "ocfd_gpu_init first"; return OCFD_ERR_STATE; }
    const long long N = L->hc.N;
    const int NS = L->NS;
    double *dp, *ddi;
    CK(cudaMallocAsync(&dp, sizeof(double) * 5 * N, L->st));
    CK(cudaMallocAsync(&ddi, sizeof(double) * NS * N, L->st));
    CK(cudaMemcpyAsync(dp, prim5, sizeof(double) * 5 * N, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(ddi, di, sizeof(double) * NS * N, cudaMemcpyHostToDevice, L->st));
    NS_DISPATCH(NS, {
      k_init_state<NSV><<<nblk(N, 256), 256, 0, L->st>>>(dp, ddi, L->f, L->d, L->u, L->v, L->w, L->T, L->di);
      LAUNCH_CHECK();
      set_time(tt);
      prims_t<NSV>(0, 0.0);
      ocfd_bc_t<NSV>();
    });
    CK(cudaFreeAsync(dp, L->st));
    CK(cudaFreeAsync(ddi, L->st));
    L->flow_ready = true;
    return check_status();
  });
}

int ocfd_gpu_upload_state(const double* f, const double* di, const double* prims) {
  return guarded([&]() -> int {
    if (!L || !L->d) { g_err = "ocfd_gpu_init first"; return OCFD_ERR_STATE; }
    const long long N = L->hc.N, H = L->hc.H;
    CK(cudaMemcpyAsync(L->f, f, sizeof(double) * 5 * N, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(L->di, di, sizeof(double) * L->NS * H, cudaMemcpyHostToDevice, L->st));
    double* pr[7] = {L->d, L->u, L->v, L->w, L->T, L->p, L->Et[L->cur]};
    for (int m = 0; m < 7; m++)
      CK(cudaMemcpyAsync(pr[m], prims + (size_t)m * H, sizeof(double) * H, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(L->Et[1 - L->cur], prims + (size_t)6 * H, sizeof(double) * H, cudaMemcpyHostToDevice, L->st));
    CK(cudaStreamSynchronize(L->st));
    L->flow_ready = true;
    return 0;
  });
}

int ocfd_gpu_flow_advance(double dt1, double tt) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    set_time(tt);
    NS_DISPATCH(L->NS, flow_advance_t<NSV>(dt1));
    return check_status();
  });
}

int ocfd_gpu_chem_advance(double dt2, int nsub) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (!L->have_kin) { g_err = "no reaction mechanism given to ocfd_gpu_init"; return OCFD_ERR_PARAM; }
    NS_DISPATCH(L->NS, chem_t<NSV>(dt2, nsub));
    return check_status();
  });
}

}  // extern "C"

namespace {
// (re)captures the Strang step as a CUDA graph when dt, the chemistry switch or the Et buffer
// parity changed since the last capture
void ensure_graph(double dt, int if_reaction, int nsub) {
  if (L->gexec && L->g_dt == dt && L->g_ifr == if_reaction && L->g_nsub == nsub && L->g_par == L->cur &&
      L->g_mode == L->chem_mode)
    return;
  drop_graphs();
  int cur0 = L->cur;
  long long l0 = L->launches;
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(L->st, cudaStreamCaptureModeThreadLocal));
  try {
    NS_DISPATCH(L->NS, {
      flow_advance_t<NSV>(0.5 * dt);
      if (if_reaction) chem_t<NSV>(dt / nsub, nsub);
      flow_advance_t<NSV>(0.5 * dt);
    });
  } catch (...) {
    cudaStreamEndCapture(L->st, &graph);
    L->cur = cur0;
    throw;
  }
  CK(cudaStreamEndCapture(L->st, &graph));
  L->gstep = graph;
  CK(cudaGraphInstantiate(&L->gexec, graph, 0));
  L->g_dt = dt; L->g_ifr = if_reaction; L->g_nsub = nsub; L->g_par = cur0; L->g_mode = L->chem_mode;
  L->g_launches = (int)(L->launches - l0);
  L->launches = l0;
  L->cur = cur0;  // six stages: the Et buffer parity returns to its start value
}
// RUN_CHUNK steps as one graph: [k_next_ht -> step] x RUN_CHUNK, each step a child node holding a
// copy of the captured step, so that a multi-step run needs no host launch per step
constexpr int RUN_CHUNK = 16;
void ensure_chunk() {
  if (L->gchunk) return;
  cudaGraph_t cg;
  CK(cudaGraphCreate(&cg, 0));
  cudaGraphNode_t prev = nullptr;
  for (int s = 0; s < RUN_CHUNK; s++) {
    cudaKernelNodeParams kp{};
    void* args[3] = {&L->ht_seq, &L->ht_counter, &L->ht_dev};
    kp.func = (void*)k_next_ht;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    cudaGraphNode_t kn, cn;
    CK(cudaGraphAddKernelNode(&kn, cg, prev ? &prev : nullptr, prev ? 1 : 0, &kp));
    CK(cudaGraphAddChildGraphNode(&cn, cg, &kn, 1, L->gstep));
    prev = cn;
  }
  CK(cudaGraphInstantiate(&L->gchunk, cg, 0));
  CK(cudaGraphDestroy(cg));
}
}  // namespace

extern "C" {

int ocfd_gpu_step(double dt, double tt, int if_reaction, int nsub) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (if_reaction && !L->have_kin) { g_err = "no reaction mechanism given to ocfd_gpu_init"; return OCFD_ERR_PARAM; }
    if (nsub < 1) nsub = 1;
    set_time(tt);
    if (L->prof) {  // timed per kernel: plain launches
      NS_DISPATCH(L->NS, {
        flow_advance_t<NSV>(0.5 * dt);
        if (if_reaction) chem_t<NSV>(dt / nsub, nsub);
        flow_advance_t<NSV>(0.5 * dt);
      });
      return check_status();
    }
    ensure_graph(dt, if_reaction, nsub);
    CK(cudaGraphLaunch(L->gexec, L->st));
    L->launches += L->g_launches;
    return check_status();
  });
}

int ocfd_gpu_run(double dt, double tt0, int nsteps, int if_reaction, int nsub) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (if_reaction && !L->have_kin) { g_err = "no reaction mechanism given to ocfd_gpu_init"; return OCFD_ERR_PARAM; }
    if (nsteps <= 0) return 0;
    if (nsub < 1) nsub = 1;
    if (nsteps > L->ht_cap) {  // the chunk graph holds the old sequence pointer
      CK(cudaStreamSynchronize(L->st));
      if (L->gchunk) { CK(cudaGraphExecDestroy(L->gchunk)); L->gchunk = nullptr; }
      if (L->ht_seq) cudaFree(L->ht_seq);
      if (L->ht_seq_host) cudaFreeHost(L->ht_seq_host);
      const int cap = std::max(nsteps, 4096);
      CK(cudaMalloc(&L->ht_seq, sizeof(double) * cap));
      CK(cudaMallocHost(&L->ht_seq_host, sizeof(double) * cap));
      L->ht_cap = cap;
    }
    if (!L->ht_counter) CK(cudaMalloc(&L->ht_counter, sizeof(int)));
    CK(cudaStreamSynchronize(L->st));
    double tt = tt0;  // tt = tt + dt after every step (OCFD_NS_Solver.f90:46)
    for (int s = 0; s < nsteps; s++) {
      L->ht_seq_host[s] = wall_ht(tt);
      tt = tt + dt;
    }
    CK(cudaMemcpyAsync(L->ht_seq, L->ht_seq_host, sizeof(double) * nsteps, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemsetAsync(L->ht_counter, 0, sizeof(int), L->st));
    ensure_graph(dt, if_reaction, nsub);
    int s = 0;
    if (nsteps >= RUN_CHUNK) {
      ensure_chunk();
      for (; s + RUN_CHUNK <= nsteps; s += RUN_CHUNK) {
        CK(cudaGraphLaunch(L->gchunk, L->st));
        L->launches += (long long)RUN_CHUNK * (L->g_launches + 1);
      }
    }
    for (; s < nsteps; s++) {
      k_next_ht<<<1, 1, 0, L->st>>>(L->ht_seq, L->ht_counter, L->ht_dev);
      LAUNCH_CHECK();
      CK(cudaGraphLaunch(L->gexec, L->st));
      L->launches += L->g_launches + 1;
    }
    return check_status();
  });
}

int ocfd_gpu_event_record(int slot) {
  return guarded([&]() -> int {
    if (!L || slot < 0 || slot >= 16) { g_err = "event slot"; return OCFD_ERR_PARAM; }
    if (!L->uev[slot]) CK(cudaEventCreate(&L->uev[slot]));
    CK(cudaEventRecord(L->uev[slot], L->st));
    return 0;
  });
}

int ocfd_gpu_event_elapsed(int a, int b, double* ms) {
  return guarded([&]() -> int {
    if (!L || a < 0 || b < 0 || a >= 16 || b >= 16 || !L->uev[a] || !L->uev[b]) { g_err = "event slot"; return OCFD_ERR_PARAM; }
    CK(cudaEventSynchronize(L->uev[b]));
    float f = 0;
    CK(cudaEventElapsedTime(&f, L->uev[a], L->uev[b]));
    *ms = f;
    return 0;
  });
}

int ocfd_gpu_pinned_alloc(size_t bytes, void** ptr) {
  return guarded([&]() -> int {
    CK(cudaMallocHost(ptr, bytes));
    return 0;
  });
}

int ocfd_gpu_pinned_free(void* ptr) {
  return guarded([&]() -> int {
    CK(cudaFreeHost(ptr));
    return 0;
  });
}

int ocfd_gpu_step_launches(void) { return L ? L->g_launches : 0; }

int ocfd_gpu_chem_mode(int mode, double tol_T) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (mode != 0 && mode != 1) { g_err = "chemistry mode must be 0 (FP64) or 1 (gated surrogate)"; return OCFD_ERR_PARAM; }
    if (mode == 1) {
      if (!L->have_kin) { g_err = "no reaction mechanism given to ocfd_gpu_init"; return OCFD_ERR_PARAM; }
      if (!(tol_T > 0.0)) { g_err = "tol_T must be positive"; return OCFD_ERR_PARAM; }
      int rc = sg_cells_setup(L->NS, L->hc.N, tol_T);
      if (rc) { g_err = "the surrogate is not trained (or loaded) for this mechanism"; return rc == -2 ? OCFD_ERR_CUDA : OCFD_ERR_STATE; }
    }
    L->chem_mode = mode;
    return 0;
  });
}

long long ocfd_gpu_chem_surrogate_rejected(long long* reasons) { return sg_cells_rejected(reasons); }

int ocfd_gpu_download_state(double* f, double* di, double* prims) {
  return guarded([&]() -> int {
    if (!L || !L->d) { g_err = "ocfd_gpu_init first"; return OCFD_ERR_STATE; }
    const long long N = L->hc.N, H = L->hc.H;
    if (f) CK(cudaMemcpyAsync(f, L->f, sizeof(double) * 5 * N, cudaMemcpyDeviceToHost, L->st));
    if (di) CK(cudaMemcpyAsync(di, L->di, sizeof(double) * L->NS * H, cudaMemcpyDeviceToHost, L->st));
    if (prims) {
      double* pr[7] = {L->d, L->u, L->v, L->w, L->T, L->p, L->Et[L->cur]};
      for (int m = 0; m < 7; m++)
        CK(cudaMemcpyAsync(prims + (size_t)m * H, pr[m], sizeof(double) * H, cudaMemcpyDeviceToHost, L->st));
    }
    CK(cudaStreamSynchronize(L->st));
    return 0;
  });
}

int ocfd_gpu_diag_begin(void) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    async_setup();
    const long long N = L->hc.N;
    const unsigned nb = nblk(N, 256);
    if (L->sep) k_diag<true><<<nb, 256, 0, L->st>>>(L->f, L->d, L->u, L->v, L->w, L->partial, L->geo);
    else k_diag<false><<<nb, 256, 0, L->st>>>(L->f, L->d, L->u, L->v, L->w, L->partial, L->geo);
    LAUNCH_CHECK();
    k_sum_partials<2><<<1, 256, 0, L->st>>>(L->partial, (int)nb, L->diag_dev);
    LAUNCH_CHECK();
    CK(cudaEventRecord(L->diag_ready, L->st));
    CK(cudaStreamWaitEvent(L->cst, L->diag_ready, 0));
    CK(cudaMemcpyAsync(L->diag_host, L->diag_dev, sizeof(double) * 2, cudaMemcpyDeviceToHost, L->cst));
    CK(cudaEventRecord(L->diag_done, L->cst));
    L->diag_pending = true;
    return 0;
  });
}

int ocfd_gpu_diag_end(double* e_mean, double* k_mean) {
  return guarded([&]() -> int {
    if (!L || !L->diag_pending) { g_err = "no ocfd_gpu_diag_begin pending"; return OCFD_ERR_STATE; }
    CK(cudaEventSynchronize(L->diag_done));
    L->diag_pending = false;
    const double nn = (double)L->P.nx * L->P.ny * L->P.nz;
    if (e_mean) *e_mean = L->diag_host[0] / nn;
    if (k_mean) *k_mean = L->diag_host[1] / nn;
    return check_status();
  });
}

int ocfd_gpu_diag(double* e_mean, double* k_mean) {
  int rc = ocfd_gpu_diag_begin();
  return rc != 0 ? rc : ocfd_gpu_diag_end(e_mean, k_mean);
}

int ocfd_gpu_snapshot(int istep, double tt) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    async_setup();
    int slot = -1;  // a free slot, else the older of the handed-out ones
    for (int m = 0; m < 2 && slot < 0; m++)
      if (L->snap_state[m] == 0) slot = m;
    if (slot < 0)
      for (int m = 0; m < 2; m++)
        if (L->snap_state[m] == 2 && (slot < 0 || L->snap_seq[m] < L->snap_seq[slot])) slot = m;
    if (slot < 0) { g_err = "two snapshots in flight: call ocfd_gpu_snapshot_wait first"; return OCFD_ERR_STATE; }
    const long long N = L->hc.N;
    const size_t n = (size_t)(5 + L->NS) * N;
    if (!L->snap_dev[slot]) {
      CK(cudaMalloc(&L->snap_dev[slot], sizeof(double) * n));
      CK(cudaMallocHost(&L->snap_host[slot], sizeof(double) * n));
    }
    k_pack_snapshot<<<nblk(N, 256), 256, 0, L->st>>>(L->d, L->u, L->v, L->w, L->T, L->di, L->NS, L->snap_dev[slot]);
    LAUNCH_CHECK();
    CK(cudaEventRecord(L->snap_ready[slot], L->st));
    CK(cudaStreamWaitEvent(L->cst, L->snap_ready[slot], 0));
    CK(cudaMemcpyAsync(L->snap_host[slot], L->snap_dev[slot], sizeof(double) * n, cudaMemcpyDeviceToHost, L->cst));
    CK(cudaEventRecord(L->snap_done[slot], L->cst));
    L->snap_state[slot] = 1;
    L->snap_seq[slot] = ++L->snap_counter;
    L->snap_istep[slot] = istep;
    L->snap_tt[slot] = tt;
    return 0;
  });
}

int ocfd_gpu_snapshot_wait(int* istep, double* tt, const double** fields) {
  return guarded([&]() -> int {
    if (!L) { g_err = "not initialised"; return OCFD_ERR_STATE; }
    int slot = -1;
    for (int m = 0; m < 2; m++)
      if (L->snap_state[m] == 1 && (slot < 0 || L->snap_seq[m] < L->snap_seq[slot])) slot = m;
    if (slot < 0) { g_err = "no snapshot in flight"; return OCFD_ERR_STATE; }
    CK(cudaEventSynchronize(L->snap_done[slot]));
    L->snap_state[slot] = 2;
    if (istep) *istep = L->snap_istep[slot];
    if (tt) *tt = L->snap_tt[slot];
    if (fields) *fields = L->snap_host[slot];
    return 0;
  });
}

int ocfd_gpu_download_rhybrid(double* r) {
  return guarded([&]() -> int {
    if (!L || !L->d) { g_err = "ocfd_gpu_init first"; return OCFD_ERR_STATE; }
    CK(cudaMemcpyAsync(r, L->Rh, sizeof(double) * L->hc.H, cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    return 0;
  });
}

int ocfd_gpu_download_metrics(double* m) {
  return guarded([&]() -> int {
    if (!L || !L->d) { g_err = "ocfd_gpu_init first"; return OCFD_ERR_STATE; }
    const long long H = L->hc.H;
    if (L->sep) {
      double* tmp;
      CK(cudaMalloc(&tmp, sizeof(double) * 10 * H));
      k_expand_metrics<<<nblk(H, 256), 256, 0, L->st>>>(L->geo, tmp, H);
      LAUNCH_CHECK();
      CK(cudaMemcpyAsync(m, tmp, sizeof(double) * 10 * H, cudaMemcpyDeviceToHost, L->st));
      CK(cudaStreamSynchronize(L->st));
      CK(cudaFree(tmp));
      return 0;
    }
    for (int mm = 0; mm < 10; mm++) CK(cudaMemcpy(m + mm * H, L->met[mm], sizeof(double) * H, cudaMemcpyDeviceToHost));
    return 0;
  });
}

int ocfd_gpu_chem_setup(const ocfd_thermo* th, const ocfd_kinetics* kin, int realgas, int timeadv) {
  return guarded([&]() -> int {
    if (!th || !kin) { g_err = "null argument"; return OCFD_ERR_PARAM; }
    if (th->n_spec < 1 || th->n_spec > 9 || kin->n_spec != th->n_spec || kin->n_reac > OCFD_MAX_REAC) {
      g_err = "N_SPEC must be 1..9 and match the mechanism";
      return OCFD_ERR_PARAM;
    }
    if (!(timeadv == 1 || timeadv == 2 || timeadv == 3 || timeadv == -1)) { g_err = "CHEM_TimeAdv"; return OCFD_ERR_PARAM; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { g_err = "no CUDA device"; return OCFD_ERR_CUDA; }
    if (!L) {
      L = new Lib();
      CK(cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking));
      CK(cudaMallocHost(&L->shost, sizeof(DevStatus)));
      CK(cudaMallocHost(&L->ht_host, sizeof(double)));
    }
    L->NS = th->n_spec;
    fill_thermo(L->hc, th, realgas);
    fill_kin(L->hc, kin);
    L->hc.timeadv = timeadv;
    L->hc.ns = th->n_spec;
    L->hc.const_p = 0;  // the reference's constant-volume reactor unless ocfd_gpu_chem_constant_pressure(1)
    L->have_kin = true;
    CK(cudaMemcpyToSymbol(cC, &L->hc, sizeof(DevConst)));
    return 0;
  });
}

int ocfd_gpu_chem_batch_device(int n, double* d_di, double* d_e, const double* d_dt, const int* d_nsub) {
  return guarded([&]() -> int {
    if (!L || !L->have_kin) { g_err = "ocfd_gpu_init or ocfd_gpu_chem_setup with a mechanism first"; return OCFD_ERR_STATE; }
    if (n < 0) { g_err = "ocfd_gpu_chem_batch_device: n = " + std::to_string(n) + " must be >= 0"; return OCFD_ERR_PARAM; }
    L->b_last[0] = L->b_last[1] = 0;
    if (n == 0) return 0;
    const int nbins = 1024;
    if ((size_t)n > L->b_cap) {
      if (L->b_di) cudaFree(L->b_di);
      size_t bytes = sizeof(int) * ((size_t)n + nbins + 64);
      CK(cudaMalloc(&L->b_di, bytes));
      L->b_perm = reinterpret_cast<int*>(L->b_di);
      L->b_hist = L->b_perm + n;
      L->b_counter = L->b_hist + nbins;
      L->b_nfail = L->b_counter + 32;
      L->b_cap = n;
    }
    CK(cudaMemsetAsync(L->b_hist, 0, sizeof(int) * (nbins + 64), L->st));
    {
      KTimer t(KC_CHEM);
      k_nsub_hist<<<nblk(n, 256), 256, 0, L->st>>>(n, d_nsub, L->b_hist, nbins);
      k_nsub_scan<<<1, 32, 0, L->st>>>(L->b_hist, nbins);
      k_nsub_scatter<<<nblk(n, 256), 256, 0, L->st>>>(n, d_nsub, L->b_hist, nbins, L->b_perm);
      LAUNCH_CHECK();
    }
    int dev = 0, sms = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    {
      KTimer t(KC_CHEM);
      launch_chem_batch(L->NS, sms, n, d_di, d_e, d_dt, d_nsub, L->b_perm, L->b_counter, L->b_nfail, L->st);
      LAUNCH_CHECK();
    }
    CK(cudaMemcpyAsync(L->b_last, L->b_nfail, 2 * sizeof(int), cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    prof_collect();
    return batch_result();
  });
}

}  // extern "C"

// ---------------------------------------------------------------- batched chemistry, no allocation
// Some callers cannot let a library allocate device memory: a host application that owns the
// whole device memory budget through its own pool (the usual situation when the chemistry is
// embedded in a larger solver or a serving process), or code that must not allocate between its
// setup and its launches. ocfd_gpu_chem_batch_device gets its scratch (the sub-step ordering of
// the reactors, the histogram of sub-step counts and the work-queue counter) from cudaMalloc the
// first time and whenever n grows; this variant takes it from a fixed array of the library
// instead, so it allocates nothing. The array is sized for OCFD_NOALLOC_MAX_REACTORS reactors and
// lives on every GPU that loads the library until the process exits.
#define OCFD_NOALLOC_MAX_REACTORS (1 << 20)
#define OCFD_NOALLOC_BINS 1024
#define OCFD_NOALLOC_WORDS (OCFD_NOALLOC_MAX_REACTORS + OCFD_NOALLOC_BINS + 64)
static __device__ __align__(256) int g_noalloc_scratch[OCFD_NOALLOC_WORDS];

namespace {
// device address of g_noalloc_scratch per device, looked up once per device with that device
// current (in host code the array's name is only a host-side stand-in)
int* g_noalloc_ptr[64] = {};

int* noalloc_scratch() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw CudaError(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e), OCFD_ERR_CUDA);
    g_noalloc_ptr[dev] = static_cast<int*>(p);
  }
  return g_noalloc_ptr[dev];
}
}  // namespace

extern "C" {

int ocfd_gpu_chem_batch_noalloc(int n, double* d_di, double* d_e, const double* d_dt, const int* d_nsub) {
  return guarded([&]() -> int {
    if (!L || !L->have_kin) { g_err = "ocfd_gpu_init or ocfd_gpu_chem_setup with a mechanism first"; return OCFD_ERR_STATE; }
    if (n < 0) {
      g_err = "ocfd_gpu_chem_batch_noalloc: n = " + std::to_string(n) + " must be >= 0";
      return OCFD_ERR_PARAM;
    }
    if (n > OCFD_NOALLOC_MAX_REACTORS) {
      g_err = "ocfd_gpu_chem_batch_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch of " +
              std::to_string(OCFD_NOALLOC_MAX_REACTORS) + " reactors (use ocfd_gpu_chem_batch_device)";
      return OCFD_ERR_PARAM;
    }
    L->b_last[0] = L->b_last[1] = 0;
    if (n == 0) return 0;
    int* perm = noalloc_scratch();
    int* hist = perm + OCFD_NOALLOC_MAX_REACTORS;
    int* counter = hist + OCFD_NOALLOC_BINS;
    int* nfail = counter + 32;
    // the array keeps the previous call's contents: the histogram and the counters restart at 0
    CK(cudaMemsetAsync(hist, 0, sizeof(int) * (OCFD_NOALLOC_BINS + 64), L->st));
    {
      KTimer t(KC_CHEM);
      k_nsub_hist<<<nblk(n, 256), 256, 0, L->st>>>(n, d_nsub, hist, OCFD_NOALLOC_BINS);
      k_nsub_scan<<<1, 32, 0, L->st>>>(hist, OCFD_NOALLOC_BINS);
      k_nsub_scatter<<<nblk(n, 256), 256, 0, L->st>>>(n, d_nsub, hist, OCFD_NOALLOC_BINS, perm);
      LAUNCH_CHECK();
    }
    int dev = 0, sms = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    {
      KTimer t(KC_CHEM);
      launch_chem_batch(L->NS, sms, n, d_di, d_e, d_dt, d_nsub, perm, counter, nfail, L->st);
      LAUNCH_CHECK();
    }
    CK(cudaMemcpyAsync(L->b_last, nfail, 2 * sizeof(int), cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    prof_collect();
    return batch_result();
  });
}

int ocfd_gpu_chem_batch(int n, double* di, double* e, const double* dt, const int* nsub) {
  return guarded([&]() -> int {
    if (!L || !L->have_kin) { g_err = "ocfd_gpu_init or ocfd_gpu_chem_setup with a mechanism first"; return OCFD_ERR_STATE; }
    if (n < 0) { g_err = "ocfd_gpu_chem_batch: n = " + std::to_string(n) + " must be >= 0"; return OCFD_ERR_PARAM; }
    L->b_last[0] = L->b_last[1] = 0;
    if (n == 0) return 0;
    const int NS = L->NS;
    double *ddi, *de, *ddt;
    int* dns = nullptr;
    CK(cudaMallocAsync(&ddi, sizeof(double) * (size_t)n * NS, L->st));
    CK(cudaMallocAsync(&de, sizeof(double) * n, L->st));
    CK(cudaMallocAsync(&ddt, sizeof(double) * n, L->st));
    if (nsub) CK(cudaMallocAsync(&dns, sizeof(int) * n, L->st));
    CK(cudaMemcpyAsync(ddi, di, sizeof(double) * (size_t)n * NS, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(de, e, sizeof(double) * n, cudaMemcpyHostToDevice, L->st));
    CK(cudaMemcpyAsync(ddt, dt, sizeof(double) * n, cudaMemcpyHostToDevice, L->st));
    if (nsub) CK(cudaMemcpyAsync(dns, nsub, sizeof(int) * n, cudaMemcpyHostToDevice, L->st));
    int rc = ocfd_gpu_chem_batch_device(n, ddi, de, ddt, dns);
    if (rc != 0 && rc != OCFD_ERR_CHEM) return rc;
    CK(cudaMemcpyAsync(di, ddi, sizeof(double) * (size_t)n * NS, cudaMemcpyDeviceToHost, L->st));
    CK(cudaMemcpyAsync(e, de, sizeof(double) * n, cudaMemcpyDeviceToHost, L->st));
    CK(cudaFreeAsync(ddi, L->st));
    CK(cudaFreeAsync(de, L->st));
    CK(cudaFreeAsync(ddt, L->st));
    if (dns) CK(cudaFreeAsync(dns, L->st));
    CK(cudaStreamSynchronize(L->st));
    if (rc) g_err = "chemistry: " + std::to_string(L->b_last[1]) +
                    " reactor(s) with a zero Gauss pivot or a non-finite result (their values are returned as computed)";
    return rc;
  });
}

int ocfd_gpu_chem_compiled_mechanism(int on) {
  return guarded([&]() -> int {
    if (!L || !L->have_kin) { g_err = "ocfd_gpu_init or ocfd_gpu_chem_setup with a mechanism first"; return OCFD_ERR_STATE; }
    if (on >= 0) L->mech_on = on != 0;
    return L->hc.timeadv == -1 && current_mech() != 0 ? 1 : 0;
  });
}

int ocfd_gpu_chem_constant_pressure(int on) {
  return guarded([&]() -> int {
    if (!L || !L->have_kin) { g_err = "ocfd_gpu_init or ocfd_gpu_chem_setup with a mechanism first"; return OCFD_ERR_STATE; }
    if (on < 0) return L->hc.const_p;
    L->hc.const_p = on ? 1 : 0;
    CK(cudaMemcpyToSymbol(cC, &L->hc, sizeof(DevConst)));
    return 0;
  });
}

int ocfd_gpu_chem_batch_status(long long* newton_fail, long long* bad) {
  if (!L) return OCFD_ERR_STATE;
  if (newton_fail) *newton_fail = L->b_last[0];
  if (bad) *bad = L->b_last[1];
  return 0;
}

int ocfd_gpu_stats(long long* neg_et, long long* newton_fail) {
  return guarded([&]() -> int {
    if (!L || !L->sdev) { g_err = "not initialised"; return OCFD_ERR_STATE; }
    CK(cudaMemcpyAsync(L->shost, L->sdev, sizeof(DevStatus), cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    if (neg_et) *neg_et = (long long)L->shost->neg_total;
    if (newton_fail) *newton_fail = L->shost->newton_fail;
    return 0;
  });
}

int ocfd_gpu_filtering(int istep, int nfiltering, const double* filter, int* applied) {
  return guarded([&]() -> int {
    if (applied) *applied = 0;
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (nfiltering < 0 || nfiltering > 10 || (nfiltering > 0 && !filter)) {
      g_err = "NFiltering must be 0..10 with a Filter table";
      return OCFD_ERR_PARAM;
    }
    bool any = false;
    for (int m = 0; m < nfiltering; m++) {
      const long cad = std::lround(filter[100 * m]);
      if (cad < 1) { g_err = "filter step interval Filter(1,m) must be >= 1"; return OCFD_ERR_PARAM; }
      if (istep % cad == 0) any = true;
    }
    if (!any) return 0;
    NS_DISPATCH(L->NS, filter_t<NSV>(istep, nfiltering, filter));
    if (applied) *applied = 1;
    return check_status();
  });
}

int ocfd_gpu_keep_viscosity(int on) {
  return guarded([&]() -> int {
    if (!L || !L->d) { g_err = "ocfd_gpu_init first"; return OCFD_ERR_STATE; }
    const bool want = on != 0;
    if (want && L->NS == 1 && !L->amu_keep) {
      CK(cudaMalloc(&L->amu_keep, sizeof(double) * L->hc.N));
      CK(cudaMemsetAsync(L->amu_keep, 0, sizeof(double) * L->hc.N, L->st));
    }
    if (L->keep_amu != want) {
      L->keep_amu = want;
      drop_graphs();
    }
    return 0;
  });
}

int ocfd_gpu_ana_box(double tt, double* out) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (!out) { g_err = "out is NULL"; return OCFD_ERR_PARAM; }
    if (L->NS == 1 && !L->keep_amu) {
      g_err = "ana_box averages the stage viscosity: call ocfd_gpu_keep_viscosity(1) before the steps";
      return OCFD_ERR_STATE;
    }
    const long long N = L->hc.N;
    const unsigned nb = nblk(N, 256);
    double* part = ana_partials((size_t)13 * nb);
    exchange({L->u}, 7);  // exchange_boundary_xyz(u) (OCFD_ANA.f90:214)
    const double* amu = L->NS == 1 ? L->amu_keep : L->amu;
    if (L->sep) k_ana_box<true><<<nb, 256, 0, L->st>>>(L->d, L->u, L->v, L->w, L->T, L->p, L->Et[L->cur], amu, part, L->geo);
    else k_ana_box<false><<<nb, 256, 0, L->st>>>(L->d, L->u, L->v, L->w, L->T, L->p, L->Et[L->cur], amu, part, L->geo);
    LAUNCH_CHECK();
    std::vector<double> h((size_t)13 * nb);
    CK(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    double sm[13] = {};
    for (unsigned b = 0; b < nb; b++)
      for (int m = 0; m < 13; m++) sm[m] = sm[m] + h[(size_t)13 * b + m];
    const double nn = (double)L->P.nx * L->P.ny * L->P.nz;
    for (double& x : sm) x = x / nn;
    k_ana_drms<<<nb, 256, 0, L->st>>>(L->d, sm[6], part);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(h.data(), part, sizeof(double) * nb, cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    double drs = 0.0;
    for (unsigned b = 0; b < nb; b++) drs = drs + h[b];
    // OCFD_ANA.f90:260-286
    double u_rms = sm[0], v_rms = sm[1], w_rms = sm[2], ux_rms = sm[3], ux_sk = sm[4], ux_fl = sm[5];
    const double d_aver = sm[6], c_aver = sm[7], amu_aver = sm[8], ek = sm[9], T_aver = sm[10];
    double u_sk = sm[11], u_fl = sm[12];
    const double vv_rms = std::sqrt((u_rms + v_rms + w_rms) / 3.0);
    const double amt = std::sqrt(u_rms + v_rms + w_rms) / c_aver;
    u_rms = std::sqrt(u_rms); v_rms = std::sqrt(v_rms); w_rms = std::sqrt(w_rms); ux_rms = std::sqrt(ux_rms);
    const double alamda = vv_rms / ux_rms, alamdax = u_rms / ux_rms;
    const double re_l = vv_rms * alamda * d_aver / amu_aver, re_lx = vv_rms * alamdax * d_aver / amu_aver;
    ux_sk = ux_sk / hp3(ux_rms); ux_fl = ux_fl / hp4(ux_rms);
    u_sk = u_sk / hp3(u_rms); u_fl = u_fl / hp4(u_rms);
    const double d_rms = std::sqrt(drs / nn);
    const double o[19] = {tt, re_l, re_lx, amt, vv_rms, u_rms, v_rms, w_rms, u_sk, u_fl, ux_sk, ux_fl, ek, d_rms,
                          T_aver, amu_aver, d_aver, ux_rms, alamdax};
    for (int m = 0; m < 19; m++) out[m] = o[m];
    return check_status();
  });
}

int ocfd_gpu_ana_q(double* q) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (!q) { g_err = "q is NULL"; return OCFD_ERR_PARAM; }
    const long long N = L->hc.N;
    exchange({L->u, L->v, L->w}, 7);
    // du is scratch between steps
    if (L->sep) k_ana_q<true><<<nblk(N, 256), 256, 0, L->st>>>(L->u, L->v, L->w, L->du, L->geo);
    else k_ana_q<false><<<nblk(N, 256), 256, 0, L->st>>>(L->u, L->v, L->w, L->du, L->geo);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(q, L->du, sizeof(double) * N, cudaMemcpyDeviceToHost, L->st));
    CK(cudaStreamSynchronize(L->st));
    return 0;
  });
}

int ocfd_gpu_ana_time_average(double dt, int* k_average, double* t_average) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    const long long N = L->hc.N;
    const size_t n = (size_t)(5 + L->NS) * N;
    if (!L->avg) {  // first call with nothing uploaded: start from zero (:80-88)
      CK(cudaMalloc(&L->avg, sizeof(double) * n));
      CK(cudaMemsetAsync(L->avg, 0, sizeof(double) * n, L->st));
      L->k_average = 0;
      L->t_average = 0.0;
    }
    const double K = (double)L->k_average;
    NS_DISPATCH(L->NS, (k_ana_average<NSV><<<nblk(N, 256), 256, 0, L->st>>>(L->d, L->u, L->v, L->w, L->T, L->di,
                                                                              L->avg, K)));
    LAUNCH_CHECK();
    L->k_average = L->k_average + 1;
    L->t_average = L->t_average + dt;
    if (k_average) *k_average = L->k_average;
    if (t_average) *t_average = L->t_average;
    return 0;
  });
}

int ocfd_gpu_ana_average(int upload, double* fields, int* k_average, double* t_average) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    const size_t n = (size_t)(5 + L->NS) * L->hc.N;
    if (upload) {
      if (!fields || !k_average || !t_average) { g_err = "upload needs fields, K_average and t_average"; return OCFD_ERR_PARAM; }
      if (!L->avg) CK(cudaMalloc(&L->avg, sizeof(double) * n));
      CK(cudaMemcpyAsync(L->avg, fields, sizeof(double) * n, cudaMemcpyHostToDevice, L->st));
      CK(cudaStreamSynchronize(L->st));
      L->k_average = *k_average;
      L->t_average = *t_average;
      return 0;
    }
    if (!L->avg) { g_err = "no time average accumulated"; return OCFD_ERR_STATE; }
    if (fields) {
      CK(cudaMemcpyAsync(fields, L->avg, sizeof(double) * n, cudaMemcpyDeviceToHost, L->st));
      CK(cudaStreamSynchronize(L->st));
    }
    if (k_average) *k_average = L->k_average;
    if (t_average) *t_average = L->t_average;
    return 0;
  });
}

int ocfd_gpu_set_tiles(const int* choice) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (!choice) { g_err = "choice is NULL"; return OCFD_ERR_PARAM; }
    for (int d = 0; d < 3; d++)
      if (choice[d] < 0 || choice[d] >= FLUX_TILE_SHAPES) { g_err = "flux tile shape must be 0, 1 or 2"; return OCFD_ERR_PARAM; }
    if (L->P.if_scheme_character == 1 && (choice[0] | choice[1] | choice[2]) != 0) {
      g_err = "the characteristic flux has one tile shape (0)";
      return OCFD_ERR_PARAM;
    }
    if (choice[3] < 1 || choice[4] < 0) {
      g_err = "k planes per block must be >= 1 (k_visc_div: >= 0, 0 = per-cell form)";
      return OCFD_ERR_PARAM;
    }
    for (int m = 5; m < 8; m++)
      if (choice[m] != 0 && choice[m] != 1) {
        g_err = "metric forms must be 0 or 1";
        return OCFD_ERR_PARAM;
      }
    if (choice[8] < 0 || choice[8] > 3) {
      g_err = "the stream switches (choice[8]) must be 0..3";
      return OCFD_ERR_PARAM;
    }
    apply_tiles(choice);
    return 0;
  });
}

int ocfd_gpu_get_tiles(int* choice) {
  if (!L || !choice) return OCFD_ERR_STATE;
  for (int d = 0; d < 3; d++) choice[d] = L->flux_ts[d];
  choice[3] = L->kc_ev;
  choice[4] = L->kc_div;
  choice[5] = L->sep ? (int)L->met_flux : 1;
  choice[6] = L->sep ? (int)L->met_ev : 1;
  choice[7] = L->sep ? (int)L->met_div : 1;
  choice[8] = (int)L->fork_visc | (int)L->fork_species << 1;
  return 0;
}

int ocfd_gpu_autotune(int reps, int* choice, double* ms) {
  return guarded([&]() -> int {
    if (!L || !L->flow_ready) { g_err = "state not initialised"; return OCFD_ERR_STATE; }
    if (reps < 0) { g_err = "reps must be >= 0"; return OCFD_ERR_PARAM; }
    int best[TUNE_N];
    double t[TUNE_TIMES];
    const std::string key = tune_key();
    auto it = g_tune_cache.find(key);
    if (reps == 0 && it != g_tune_cache.end()) {
      for (int m = 0; m < TUNE_N; m++) best[m] = it->second[m];
      for (int m = 0; m < TUNE_TIMES; m++) t[m] = -1.0;
    } else {
      NS_DISPATCH(L->NS, tune_t<NSV>(reps > 0 ? reps : 3, best, t));
      std::array<int, TUNE_N> a;
      for (int m = 0; m < TUNE_N; m++) a[m] = best[m];
      g_tune_cache[key] = a;
    }
    apply_tiles(best);
    if (choice)
      for (int m = 0; m < TUNE_N; m++) choice[m] = best[m];
    if (ms)
      for (int m = 0; m < TUNE_TIMES; m++) ms[m] = t[m];
    return check_status();
  });
}

int ocfd_gpu_profile(int enable) {
  if (!L) return OCFD_ERR_STATE;
  L->prof = enable != 0;
  for (int c = 0; c < KC_NUM; c++) { L->kc_ms[c] = 0; L->kc_n[c] = 0; }
  return 0;
}
int ocfd_gpu_profile_read(int cls, double* ms, long long* count) {
  if (!L || cls < 0 || cls >= KC_NUM) return OCFD_ERR_PARAM;
  *ms = L->kc_ms[cls];
  *count = L->kc_n[cls];
  return 0;
}
const char* ocfd_gpu_profile_name(int cls) { return (cls >= 0 && cls < KC_NUM) ? kc_names[cls] : ""; }
int ocfd_gpu_profile_nclass(void) { return KC_NUM; }
void* ocfd_gpu_stream(void) { return L ? (void*)L->st : nullptr; }
long long ocfd_gpu_launch_count(void) { return L ? (long long)L->launches : 0; }
int ocfd_gpu_is_separable(void) { return L && L->sep ? 1 : 0; }
long long ocfd_gpu_device_bytes(void) { return L ? (long long)L->arena_used : 0; }

double ocfd_gpu_fp64_peak_gflops(void) {
  double r = -1.0;
  guarded([&]() -> int {
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    double* out;
    CK(cudaMalloc(&out, sizeof(double)));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    const int iters = 1 << 14, blocks = sms * 8, threads = 256;
    k_fp64_peak<<<blocks, threads>>>(out, 64, 1.0000001, 1e-9);  // warm-up
    CK(cudaEventRecord(a));
    k_fp64_peak<<<blocks, threads>>>(out, iters, 1.0000001, 1e-9);
    CK(cudaEventRecord(b));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    r = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e9;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    return 0;
  });
  return r;
}

const char* ocfd_gpu_last_error(void) { return g_err.c_str(); }

int ocfd_gpu_finalize(void) {
  release();
  return 0;
}

}  // extern "C"
