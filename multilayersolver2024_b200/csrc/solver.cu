// solver.cu -- device-resident mesh, per-call layer description and the
// layerSolve orchestration behind the C ABI of include/mlxpbd.h.
//
// Data layout in HBM (per solver):
//   tets, colour-sorted (colour c owns [color_off[c], color_off[c+1])):
//     vid int4[T], dminv R[9][T], vol R[T], mat R[stride][T], lambda R[6][T]
//   vertices: pos R4[N] = (x, y, z, 1/m), oldp/xprev/resv R4[N],
//     vmass double[N], ri double4[N] (FP64 body-frame offsets)
//   bodies: Body[nb] (FP64)
// Host-side per-layer preprocessing builds CSR lists (elastic tets per colour,
// vertices / boundary vertices / rigid contacts per body, elastic contacts per
// vertex) and caches the contact-independent part across calls.
#include "../../include/mlxpbd.h"
#include "common.cuh"
#include "tet_kernels.cuh"
#include "body_kernels.cuh"
#include "persistent.cuh"
#include "cluster.cuh"
#include "groups.cuh"
#include "layers_dev.cuh"
#include "contacts.cuh"
#include "monitor.cuh"
#include "partition.h"
#include "warmstart.cuh"
#include "pcg.cuh"
#include "solver.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstddef>
#include <chrono>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace mlx;

namespace mlx {
thread_local std::string g_err;
int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace mlx

#define CU(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess)                                                                 \
      return set_error(MLX_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));    \
  } while (0)
#define CHECK(x)           \
  do {                     \
    int rc_ = (x);         \
    if (rc_ != MLX_OK) return rc_; \
  } while (0)

namespace {

// ---- conversion kernels (MATLAB layout <-> device layout) -----------------
template <typename R>
__global__ void k_load_pos(const double* __restrict__ xi, const double* __restrict__ mass,
                           R4<R>* __restrict__ pos, int N) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  pos[v] = make_r4<R>((R)xi[3 * v], (R)xi[3 * v + 1], (R)xi[3 * v + 2], (R)(1.0 / mass[3 * v]));
}
template <typename R>
__global__ void k_load_vec(const double* __restrict__ a, R4<R>* __restrict__ out, int N) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  out[v] = make_r4<R>((R)a[3 * v], (R)a[3 * v + 1], (R)a[3 * v + 2], 0);
}
template <typename R>
__global__ void k_store_pos(const R4<R>* __restrict__ pos, double* __restrict__ xi, int N) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  R4<R> p = pos[v];
  xi[3 * v] = p.x; xi[3 * v + 1] = p.y; xi[3 * v + 2] = p.z;
}
template <typename R>
__global__ void k_load_lambda(const double* __restrict__ lam, const int* __restrict__ s2e,
                              R* __restrict__ out, int T) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  int e = s2e[s];
#pragma unroll
  for (int q = 0; q < 6; ++q) out[(size_t)q * T + s] = (R)lam[e + (size_t)T * q];
}
template <typename R>
__global__ void k_store_lambda(const R* __restrict__ lam, const int* __restrict__ s2e,
                               double* __restrict__ out, int T) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  int e = s2e[s];
#pragma unroll
  for (int q = 0; q < 6; ++q) out[e + (size_t)T * q] = lam[(size_t)q * T + s];
}
template <typename R>
__global__ void k_cast(const double* __restrict__ a, R* __restrict__ out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (R)a[i];
}

inline int blocks_for(long long n, int b) { return (int)((n + b - 1) / b); }

// ---- buffers ---------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  // grow: a buffer whose size changes from call to call (contact lists)
  // takes half as much again, so a slowly growing size reallocates rarely
  int ensure(size_t n, bool grow = false) {
    if (n <= bytes && p) return MLX_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t want = std::max<size_t>(grow ? n + n / 2 : n, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) return set_error(MLX_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    bytes = want;
    return MLX_OK;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() { if (p) cudaFreeHost(p); }
  int ensure(size_t n, bool grow = false) {
    if (n <= bytes && p) return MLX_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    size_t want = std::max<size_t>(grow ? n + n / 2 : n, 256);
    cudaError_t e = cudaMallocHost(&p, want);
    if (e != cudaSuccess) return set_error(MLX_ERR_ALLOC, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
    bytes = want;
    return MLX_OK;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// memcpy between host buffers, split over up to 8 host threads when it is
// large (the staging of a call's host vectors into pinned memory and back).
static void host_copy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kGrain = size_t(512) << 10;
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(std::min<size_t>(hw, 8), bytes / kGrain);
  if (nt <= 1) {
    if (bytes) std::memcpy(dst, src, bytes);
    return;
  }
  const size_t chunk = (bytes + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  for (size_t t = 1; t < nt; ++t) {
    const size_t a = t * chunk, b = std::min(bytes, a + chunk);
    if (a >= b) continue;
    try {
      th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a); });
    } catch (const std::system_error&) {
      std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a);  // no thread to be had
    }
  }
  std::memcpy(dst, src, std::min(bytes, chunk));
  for (std::thread& x : th) x.join();
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Contact-independent part of one layer column, cached across calls.
struct LayerStatic {
  bool valid = false;
  // copies of the inputs the cache was built from
  std::vector<uint8_t> isE, isBV, isRV;
  std::vector<int32_t> rid;
  int nb = 0;
  // built
  int n_rigid_elements = 0;
  bool identity_list = false;
  std::vector<int> color_count;  // per colour: number of elastic tets
  std::vector<int> color_start;  // per colour: start in the elastic list
  std::vector<int> packed;       // body_vert_off | body_verts | bnd_off | bnd_verts | list | vert_body
  size_t o_bvo = 0, o_bv = 0, o_bo = 0, o_bnd = 0, o_list = 0, o_vb = 0, o_cstart = 0, o_ccount = 0;
  int n_bnd = 0;
  size_t o_items = 0;  // CTAs of the per-body kernels (body_kernels.cuh body_of_item)
  int n_items = 0;
  // component-group path (groups.cuh): (colour, group) ranges of the elastic tets
  bool gr_ok = false;
  int gr_one = 0;
  size_t o_goff = 0;
  std::vector<int> tile;  // block size of each colour kernel (0 = default), set by the autotuner
  // cluster kernel: (colour, part) ranges of the elastic tets, colours with work
  size_t o_cloff = 0, o_clcol = 0, o_cllb = 0;
  int cl_nC = 0, cl_max_range = 0;
  // vertex slots of the cluster kernel for this layer (see cluster.cuh)
  bool cl_ok = false;
  int cl_slots = 0, cl_lam = 0;
  size_t cl_smem = 0;
  DevBuf cl_dev;  // tsrc int4[nE] | tdst int2[nE] | vhome int[N] | home_v int[N] | home_s int[N] | home_off int[P+1]
  size_t o_tsrc = 0, o_tdst = 0, o_vhome = 0, o_hv = 0, o_hs = 0, o_hoff = 0;
  DevBuf dev;       // packed ints
  DevBuf dev_rigid; // vert_rigid bytes
};

}  // namespace

namespace mlx {

// Layer caches and body buffers one caller of the layer loop owns: the
// host-buffer layerSolve and the resident stepper each have their own, so a
// captured step graph never points at memory the other path reallocates.
struct LayerWork {
  std::vector<std::unique_ptr<LayerStatic>> cache;
  DevBuf bodies, lamB;
};

// Learned warm start of the resident stepper (warmstart.cuh).
struct WarmStartState {
  int record = 0;            // keep features and targets of every step
  int mode = 0;              // 0 off, 1 perceptron, 2 given corrections
  mlx_mlp* net = nullptr;
  int col = -1, nb = 0;
  const float* y = nullptr;  // rows of corrections (device) and their stride
  int ld = 0;
  WsStatic S{};
  double gate = 1e-3;        // fall back to the plain start above this predicted fit residual (m)
  DevBuf d_static, d_rest, d_norm, d_own, d_raw, d_feat, d_rec, d_target, d_corr, d_fallback;
  void reset() {
    record = mode = 0;
    net = nullptr;
    col = -1;
    nb = 0;
    y = nullptr;
    ld = 0;
  }
};

// Multiplier warm start of the resident stepper (warmstart.cuh): the last
// two steps' converged multipliers and how many steps they hold.
struct MultiplierWarmStart {
  int on = 0, rows = 0;
  double a = 1.0, b = 0.0;
  DevBuf d_lam1, d_lam2, d_seen;
};

// Per-call bookkeeping of the layer loop (the scalars layerSolve threads
// through projectGS, xpbdLayer3D.m:94-232).
struct RunState {
  std::vector<double> residualArray;
  double runUntil = -1;
  double sumNonMon = 0;
  int totalIterations = 0;
  long long launches = 0;  // kernels launched by the loop
};

template <typename R>
struct Solver final : SolverBase {
  int device = 0;
  cudaStream_t stream = nullptr;
  int N = 0, T = 0, C = 0, energy = 0, mat_kind = 0;
  bool damp = false;
  std::vector<int> s2e, color_off;
  std::vector<int32_t> pinned;  // 0-based DOFs
  std::vector<double> vmass_h, mass3;
  DevBuf d_vid, d_dminv, d_vol, d_mat, d_lambda, d_pos, d_oldp, d_xprev, d_resv, d_vmass, d_ri,
      d_pin_dofs, d_pinx, d_partials, d_scalar, d_stage, d_s2e, d_mass3,
      d_contacts, d_cvid, d_clam, d_cgroups;
  PinnedBuf h_stage, h_scalar, h_cstage;
  LayerWork work, sim_work;
  // mlx_layer_solve's layer loop as a CUDA graph, replayed while calls keep
  // one shape: no residual monitoring, no contact list, the same layer
  // columns, iteration counts, parameters and layer masks (so every cached
  // layer static, and with it every kernel argument, is unchanged).
  // MLXPBD_HOST_GRAPH=0 turns it off.
  struct HostGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<int> lkey;
    std::vector<unsigned char> pkey;
    long long launches = 0, iterations = 0;
  } hg;
  bool host_graph_on = true;
  void drop_host_graph() {
    if (hg.exec) cudaGraphExecDestroy(hg.exec);
    hg.exec = nullptr;
  }
  bool statics_hit(const mlx_layer_desc* ld, const LayerWork& w) const;

  ~Solver() override {
    for (cudaEvent_t e : tev) cudaEventDestroy(e);
    if (sim.graph) cudaGraphExecDestroy(sim.graph);
    if (hg.exec) cudaGraphExecDestroy(hg.exec);
    if (cs_if) cudaStreamDestroy(cs_if);
    if (cs_while) cudaStreamDestroy(cs_while);
    if (cs_ns) cudaStreamDestroy(cs_ns);
    if (stream) cudaStreamDestroy(stream);
  }

  int create(const mlx_mesh_desc* md);
  int layer_solve(const mlx_layer_desc* ld, const mlx_solve_params* P, const mlx_contacts* K,
                  const mlx_solve_inputs* in, mlx_solve_outputs* out) override;

  TetData<R> tets() const {
    TetData<R> td;
    td.vid = d_vid.as<int4>();
    td.dminv = d_dminv.as<R>();
    td.vol = d_vol.as<R>();
    td.mat = d_mat.as<R>();
    td.lambda = d_lambda.as<R>();
    td.T = T;
    return td;
  }
  R4<R>* pos() const { return d_pos.as<R4<R>>(); }

  int build_static(const mlx_layer_desc* ld, int col, LayerStatic& ls, bool capturing);
  int launch_color(int c, const LayerStatic& ls, const int* dlist, R h, int bs_override = 0,
                   const DevContacts* cc = nullptr, const int* vert_body = nullptr, double hd = 0, double cr = 0);
  // per-colour tile autotuner of the resident stepper (block size of each
  // colour kernel, chosen by timing; kept per layer column)
  static constexpr int kDefaultTile = 64;
  std::vector<std::vector<int>> tiles;  // [column][colour], 0 = default
  int sim_autotune(int reps, double* before_ms, double* after_ms) override;
  int residual(const ContactData& cd, double contact_resistance, double h, double* out,
               const DevContacts* dc = nullptr);
  // the device contacts' partial sums of the residual (stream work only)
  int contact_residual_partials(const DevContacts& dc, double contact_resistance, double h, double* partials,
                                int* nblocks);
  int norm_resv(double* out);
  int validate_layers(const mlx_layer_desc* ld, const mlx_solve_params* P);
  int upload_contacts(const mlx_contacts* K, ContactData& cd);
  int run_layers(const mlx_layer_desc* ld, const mlx_solve_params* P, const mlx_contacts* K,
                 const ContactData& cd, RunState& st, bool capturing, LayerWork& w,
                 const DevContacts& dc = DevContacts{});

  // resident stepper (one per solver)
  struct Sim {
    bool ready = false;
    mlx_layer_desc ld{};
    mlx_solve_params P{};
    double air_drag = 0;
    std::vector<int32_t> layers_map, iterations, sets, rid, nr;
    std::vector<uint8_t> isE, isR, isBV, isRV;
    cudaGraphExec_t graph = nullptr;
    long long launches_per_step = 0;
  } sim;
  DevBuf d_vel, d_pin_mask, d_gsync;
  // obstacles of the resident stepper (contacts detected on the device)
  std::vector<Obstacle> sim_obs;
  double sim_restitution = 1e-2;
  DevBuf d_obs, d_cmask, d_cverts, d_cidx, d_cscan, d_clam_dev;
  // contact_coloring: colour phase of each vertex's contacts, the step's
  // buckets and their offsets / cursors / counts
  DevBuf d_vcc, d_cbucket, d_coff, d_ccur, d_chist;
  int contact_colours();
  // pinned staging of the per-layer contact lists of mlx_layer_solve
  PinnedBuf h_cpack;
  size_t cpack_used = 0;
  // buffers of mlx_find_contacts, kept across calls (they only grow)
  DevBuf fc_ob, fc_mask, fc_verts, fc_scan, fc_x, fc_pos, fc_vid, fc_out;
  DevContacts dev_contacts() const {
    DevContacts dc{};
    dc.nobs = (int)sim_obs.size();
    if (!dc.nobs) return dc;
    dc.obs = d_obs.as<Obstacle>();
    dc.mask = d_cmask.as<unsigned>();
    dc.verts = d_cverts.as<int>();
    dc.cidx = d_cidx.as<int>();
    dc.count = d_cscan.as<int>() + blocks_for(N, 256);
    dc.obs_count = dc.count + 2;
    dc.lambda = d_clam_dev.as<double>();
    dc.colored = sim.P.contact_coloring ? 1 : 0;
    dc.C = C;
    dc.vcc = d_vcc.as<int>();
    dc.cbucket = d_cbucket.as<int>();
    dc.coff = d_coff.as<int>();
    return dc;
  }
  int detect_contacts(const R4<R>* x0);  // stream work only (captured in the step)
  // device residual monitor (monitor.cuh): conditional graph nodes
  // (d_mon: the resident stepper's, whose run-until persists across steps;
  // d_mon_ls: a layer solve replayed as a graph)
  DevBuf d_mon, d_mon_ls;
  const DevBuf* mon_active = &d_mon;
  cudaStream_t cs_if = nullptr, cs_while = nullptr;
  MonState* mon() const { return mon_active->as<MonState>(); }
  int cond_handle(cudaGraphConditionalHandle* h);
  int cond_begin(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, cudaStream_t body);
  int cond_end(cudaStream_t parent);
  int residual_dev(double* out, const DevContacts& dc);
  int norm_resv_dev(double* out);
  int sim_monitor(double* ra, int cap, int32_t* len, int32_t* total_it, double* run_until, int32_t* status) override;
  struct {
    bool valid = false, device = false;
    std::vector<double> ra;
    int total_it = 0;
  } sim_last;
  WarmStartState ws;
  // PCG on the linearly implicit system (pcg.cuh); host copies of the
  // material kept from create (sorted order), device data built on first use
  std::vector<double> pcg_G, pcg_vol, pcg_lame;
  bool pcg_ready = false, vt_ready = false;
  DevBuf d_pcg_G, d_pcg_vol, d_pcg_lame, d_pcg_vt, d_pcg_pin, d_pcg_vec, d_pcg_P, d_pcg_part, d_pcg_sc, d_pcg_res;
  int pcg_setup();
  int vt_setup();
  PcgOp vt_op(double h2);
  // Newton-PCG corrections of the last layer (pcg.cuh k_ns_*): PCG
  // iterations per correction (0: off) and Gauss-Seidel iterations between
  // corrections
  int ns_iters = 0, ns_every = 0, ns_vertex_blocks = 1;
  DevBuf d_ns_jac, d_ns_tet, d_vtpos, d_ns_nb, d_ns_pslot, d_ns_K;
  int ns_topology();
  NsBlocks ns_blocks() const;
  cudaStream_t cs_ns = nullptr;
  int ns_configure(int pcg_iterations, int every) override;
  int ns_correct(double h, long long* launches);
  int pcg_solve(double h, const double* b, int iterations, double* x, double* resvec) override;
  std::vector<double> sim_p0;  // positions given to mlx_sim_init (the rest configuration)
  int ws_configure(int record, int mode, mlx_mlp* net, double gate, const float* fmean, const float* fstd, const float* omean,
                   const float* ostd, const float* corrections, int32_t* nb) override;
  int ws_fetch(float* features, float* targets, int cap, int32_t* nb, int32_t* fallbacks) override;
  int ws_after_make_rigids(const LayerWork& w);
  int ws_after_lamb_reset(const LayerWork& w);
  MultiplierWarmStart mws;
  int mws_configure(int on, double a, double b) override;
  int mws_start();
  int find_contacts(const mlx_obstacle* obs, int nobs, const double* p, int max_contacts, int32_t* vids,
                    double* normals, double* points, double* comp, int32_t* K) override;
  int sim_set_obstacles(const mlx_obstacle* obs, int nobs, double restitution) override;
  int sim_contact_count(int32_t* n) override;
  PinnedBuf h_gsync;
  PinnedBuf h_mon;  // the device monitor's state, staged for a layer solve replayed as a graph
  long long last_launches = 0;
  // Fixed-iteration layers run as one launch per colour, each launched as a
  // programmatic dependent of the previous (off with MLXPBD_PDL=0).  The
  // persistent one-launch-per-layer kernel (MLXPBD_PERSISTENT=1; one CTA of
  // 128 threads per SM unless MLXPBD_PERSIST_CTAS says otherwise) is kept as
  // an option: on B200 its grid barrier costs more than a dependent launch.
  bool persistent = false;
  bool pdl = true;
  int persist_ctas = 0;
  int launch_persistent(const LayerStatic& ls, const int* dint, const LayerDev& L, const ContactData& cd,
                        const mlx_solve_params* P, int iterations, bool body_work, LayerWork& w);
  // Thread-block-cluster path (cluster.cuh): with MLXPBD_CLUSTER=1,
  // fixed-iteration layers run as one cluster launch each when the vertex
  // records of the mesh fit in the shared memory of a cluster
  // (MLXPBD_CLUSTER_SIZE forces the number of CTAs, a power of two up to 16).
  // Off by default: on a 98k-tet mesh one launch per colour is faster.
  bool cluster_ok = false;
  int cl_size = 0, cl_threads = 0, cl_rec_slots = 0, cl_lam_slots = 0;
  size_t cl_smem = 0;
  std::vector<int> tpart_sorted;  // part of each tet, sorted order
  std::vector<int4> vid_sorted;   // 0-based corners, sorted order
  std::vector<int> vowner;        // part owning each vertex
  long long cl_budget = 0;        // dynamic shared memory a CTA may use
  int plan_cluster(const mlx_mesh_desc* md, MeshPartition& mp);
  // Component-group path (groups.cuh): a fixed-iteration layer without rigid
  // bodies or host contacts runs as one launch, one CTA per group of
  // consecutive vertex-disconnected components (records in shared memory).
  // Chosen at mlx_create when the components are contiguous vertex and tet
  // ranges, every group fits in a CTA's shared memory and the estimated sweep
  // is shorter than with colour launches; MLXPBD_GROUPS=0 turns it off, =1
  // skips the estimate.
  bool groups_ok = false;
  int gr_G = 0;
  int gr_cs = 1;  // CTAs per group (a thread-block cluster when > 1)
  size_t gr_smem = 0;
  std::vector<int> tgroup_sorted;  // group of each tet, sorted order
  DevBuf d_gv0, d_tloc, d_gpin;
  int plan_groups(const mlx_mesh_desc* md);
  // buildLayers + findBoundaryVertices on the device (layers_dev.cuh)
  DevBuf lb_p, lb_oldp, lb_dminv, lb_norms, lb_norms_sorted, lb_elems, lb_order, lb_rank, lb_forced, lb_parent,
      lb_rep, lb_root, lb_flag, lb_scan, lb_sets, lb_key, lb_touch, lb_isE, lb_isBV, lb_isRV, lb_body, lb_small,
      lb_tmp;
  const double* lb_dminv_src = nullptr;  // host DmInv the device copy was made from
  int build_layers(const double* p, const double* oldp, double h, int ordering, const int32_t* order,
                   const double* dminv, const double* sorted_layers, int L, const uint8_t* forced, int32_t* sets,
                   int32_t* num_rigids, uint8_t* is_elastic, uint8_t* is_boundary, uint8_t* is_rigid_vertex,
                   int32_t* vertex_body) override;
  int launch_groups(const LayerStatic& ls, const int* dint, const mlx_solve_params* P, int iterations,
                    const DevContacts& dc, const HostContactGroups* hc = nullptr);
  int build_cluster_slots(LayerStatic& ls, const std::vector<int>& list);
  int launch_cluster(const LayerStatic& ls, const int* dint, const LayerDev& L, const ContactData& cd,
                     const mlx_solve_params* P, int iterations, bool body_work, LayerWork& w);
  int reset_gsync();
  int check_gsync();
  cudaLaunchConfig_t pdl_config(int grid, int block) const {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = stream;
    return cfg;
  }
  static cudaLaunchAttribute pdl_attr() {
    cudaLaunchAttribute a;
    a.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a.val.programmaticStreamSerializationAllowed = 1;
    return a;
  }
  // colour-sweep timing: an event pair around every iteration's sweep
  bool sweep_timing = false;
  std::vector<cudaEvent_t> tev;
  size_t tev_used = 0;
  std::vector<double> tev_bytes;    // algorithmic bytes of the sweep of each pair
  std::vector<long long> tev_launches;
  double sweep_ms = 0, sweep_bytes = 0;
  long long sweep_launches = 0;
  double bytes_per_tet() const;
  double group_bytes_per_tet() const;
  int record_event(cudaEvent_t e, bool capturing);
  int enable_sweep_timing(int on) override;
  int sweep_stats(double* ms, double* bytes, long long* launches, int reset) override;
  int collect_sweep_times();
  int sim_setup(const mlx_layer_desc* ld, const mlx_solve_params* P, const double* p0, const double* v0);
  int sim_issue_step(long long* launches, bool capturing);
  int sim_step(int nsteps, int use_graph, double* device_ms) override;
  int sim_add_velocity(const int32_t* dofs, const double* dv, int n) override;
  int sim_get_state(double* p, double* v) override;
  int sim_init(const mlx_layer_desc* ld, const mlx_solve_params* P, const double* p0, const double* v0,
               double air_drag) override {
    sim.air_drag = air_drag;
    return sim_setup(ld, P, p0, v0);
  }
  long long sim_launches_per_step() const override { return sim.launches_per_step; }
  std::string launch_path() const override {
    if (persistent) return "persistent cooperative kernel per layer (" + std::to_string(persist_ctas) + " CTAs)";
    if (groups_ok && !cluster_ok && gr_cs > 1)
      return "body-free layers: one launch, " + std::to_string(gr_G) + " clusters of " + std::to_string(gr_cs) +
             " CTAs each owning whole components (records in distributed shared memory); other layers: one launch "
             "per colour (programmatic dependent launches)";
    if (groups_ok && !cluster_ok)
      return "body-free layers: one launch, " + std::to_string(gr_G) + " CTAs each owning whole components "
             "(records in shared memory); other layers: one launch per colour (programmatic dependent launches)";
    if (cluster_ok)
      return "cluster kernel per layer: " + std::to_string(cl_size) + " CTAs x " + std::to_string(cl_threads) +
             " threads, vertex slots" + (cl_lam_slots ? " and multipliers" : "") + " in shared memory";
    std::string t;
    if (!tiles.empty()) {
      int lo = 1 << 30, hi = 0;
      for (const auto& v : tiles)
        for (int b : v)
          if (b > 0) { lo = std::min(lo, b); hi = std::max(hi, b); }
      if (hi > 0) t = ", autotuned tiles " + std::to_string(lo) + "-" + std::to_string(hi) + " threads";
    }
    return std::string("one launch per colour") + (pdl ? " (programmatic dependent launches)" : "") + t;
  }
  long long launches_last_call() const override { return last_launches; }
};

template <typename R>
int Solver<R>::create(const mlx_mesh_desc* md) {
  N = md->num_vertices;
  T = md->num_tets;
  C = md->num_colors;
  energy = md->energy_type;
  device = md->device;
  if (N <= 0 || T <= 0 || C <= 0) return set_error(MLX_ERR_ARGUMENT, "mesh needs N, T, num_colors > 0");
  if (!md->t || !md->mass || !md->DmInv || !md->volume || !md->element_color)
    return set_error(MLX_ERR_ARGUMENT, "mesh arrays t, mass, DmInv, volume, element_color are required");
  if (md->num_pinned_dofs > 0 && !md->pinned_dofs) return set_error(MLX_ERR_ARGUMENT, "pinned_dofs is NULL");
  // colour validity: every colour id in range and no two tets of one colour share a vertex
  std::vector<int> cnt(C + 1, 0);
  for (int e = 0; e < T; ++e) {
    int c = md->element_color[e];
    if (c < 1 || c > C) return set_error(MLX_ERR_ARGUMENT, "element_color out of [1, num_colors]");
    ++cnt[c];
    for (int k = 0; k < 4; ++k) {
      int v = md->t[e + (size_t)T * k];
      if (v < 1 || v > N) return set_error(MLX_ERR_ARGUMENT, "tet vertex index out of range");
    }
  }
  {
    std::vector<int> last(N, -1);  // last colour that touched a vertex, per colour pass
    std::vector<std::vector<int>> byc(C + 1);
    for (int e = 0; e < T; ++e) byc[md->element_color[e]].push_back(e);
    for (int c = 1; c <= C; ++c)
      for (int e : byc[c])
        for (int k = 0; k < 4; ++k) {
          int v = md->t[e + (size_t)T * k] - 1;
          if (last[v] == c) return set_error(MLX_ERR_ARGUMENT, "element_color is not a valid colouring");
          last[v] = c;
        }
  }
  // material encoding
  if (energy == MLX_ENERGY_NEOHOOKEAN) {
    if (!md->mu || !md->lambda) return set_error(MLX_ERR_ARGUMENT, "Neo-Hookean mesh needs mu and lambda");
    for (int e = 0; e < T; ++e)
      if (!(md->mu[e] > 0) || !(md->volume[e] > 0))
        return set_error(MLX_ERR_ARGUMENT, "Neo-Hookean mesh needs mu > 0 and volume > 0 for every tet");
    mat_kind = MAT_NH;
    damp = false;
  } else if (energy == MLX_ENERGY_STVK_VOIGT) {
    if (md->alpha && md->beta) {
      mat_kind = MAT_STVK_BLOCKS;
      damp = false;
      for (int e = 0; e < T; ++e) {
        const double* a = md->alpha + 36 * (size_t)e;
        const double* b = md->beta + 36 * (size_t)e;
        for (int r = 0; r < 6; ++r)
          for (int c = 0; c < 6; ++c) {
            bool top = r < 3 && c < 3, diag = r >= 3 && r == c;
            if (!top && !diag && (a[r + 6 * c] != 0.0 || b[r + 6 * c] != 0.0))
              return set_error(MLX_ERR_UNSUPPORTED,
                               "alpha/beta must be block diagonal (3x3 (+) diagonal 3x3) as Mesh3D.updateMaterials builds them");
          }
        for (int i = 0; i < 36; ++i)
          if (b[i] != 0.0) damp = true;
      }
    } else if (md->mu && md->lambda) {
      mat_kind = MAT_STVK_LAME;
      damp = false;
      if (md->alpha1)
        for (int e = 0; e < T; ++e)
          if (md->alpha1[e] != 0.0) damp = true;
    } else {
      return set_error(MLX_ERR_ARGUMENT, "StVK mesh needs alpha/beta or mu/lambda");
    }
  } else {
    return set_error(MLX_ERR_ARGUMENT, "unknown energy_type");
  }
  for (int i = 0; i < md->num_pinned_dofs; ++i) {
    int d = md->pinned_dofs[i] - 1;
    if (d < 0 || d >= 3 * N) return set_error(MLX_ERR_ARGUMENT, "pinned DOF out of range");
    pinned.push_back(d);
  }
  mass3.assign(md->mass, md->mass + 3 * (size_t)N);
  vmass_h.resize(N);
  for (int v = 0; v < N; ++v) {
    double m = md->mass[3 * v];
    if (!(m > 0)) return set_error(MLX_ERR_ARGUMENT, "vertex masses must be positive");
    vmass_h[v] = m;
  }

  DeviceGuard g(device);
  color_off.assign(C + 1, 0);
  for (int c = 1; c <= C; ++c) color_off[c] = color_off[c - 1] + cnt[c];
  MeshPartition mp;
  CHECK(plan_cluster(md, mp));
  // sorted order: by colour, then (cluster path) by part, then element id.
  // Tets of one colour share no vertex, so their order changes no result.
  s2e.assign(T, 0);
  {
    std::vector<int> fill(color_off.begin(), color_off.end() - 1);
    if (cluster_ok) {
      const int P = cl_size;
      std::vector<int> cp((size_t)C * P + 1, 0);
      for (int e = 0; e < T; ++e) ++cp[(size_t)(md->element_color[e] - 1) * P + mp.tpart[e] + 1];
      for (size_t q = 1; q < cp.size(); ++q) cp[q] += cp[q - 1];
      for (int e = 0; e < T; ++e) s2e[cp[(size_t)(md->element_color[e] - 1) * P + mp.tpart[e]]++] = e;
      tpart_sorted.assign(T, 0);
      for (int s = 0; s < T; ++s) tpart_sorted[s] = mp.tpart[s2e[s]];
    } else {
      for (int e = 0; e < T; ++e) s2e[fill[md->element_color[e] - 1]++] = e;
    }
  }

  // ---- host-side packing of the rest data in sorted order ----
  const int stride = mat_stride(mat_kind);
  std::vector<int4> vid(T);
  std::vector<R> dminv(9 * (size_t)T), vol(T), mat((size_t)stride * T);
  for (int s = 0; s < T; ++s) {
    int e = s2e[s];
    vid[s] = make_int4(md->t[e] - 1, md->t[e + (size_t)T] - 1, md->t[e + 2 * (size_t)T] - 1,
                       md->t[e + 3 * (size_t)T] - 1);
    for (int j = 0; j < 9; ++j) dminv[(size_t)j * T + s] = (R)md->DmInv[9 * (size_t)e + j];
    vol[s] = (R)md->volume[e];
    if (mat_kind == MAT_STVK_BLOCKS) {
      const double* a = md->alpha + 36 * (size_t)e;
      const double* b = md->beta + 36 * (size_t)e;
      double ab[36];
      for (int c = 0; c < 6; ++c)
        for (int r = 0; r < 6; ++r) {
          double acc = 0;
          for (int k = 0; k < 6; ++k) acc += a[r + 6 * k] * b[k + 6 * c];
          ab[r + 6 * c] = acc;
        }
      for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) {
          mat[(size_t)(r + 3 * c) * T + s] = (R)a[r + 6 * c];
          mat[(size_t)(12 + r + 3 * c) * T + s] = (R)ab[r + 6 * c];
        }
      for (int q = 0; q < 3; ++q) {
        mat[(size_t)(9 + q) * T + s] = (R)a[(3 + q) + 6 * (3 + q)];
        mat[(size_t)(21 + q) * T + s] = (R)ab[(3 + q) + 6 * (3 + q)];
      }
    } else if (mat_kind == MAT_NH) {
      const double v = md->volume[e], mu = md->mu[e], lm = md->lambda[e];
      mat[s] = (R)(1.0 / (v * mu));
      mat[(size_t)T + s] = (R)(lm > mu ? 1.0 / (v * (lm - mu)) : 0.0);
    } else {
      mat[s] = (R)md->mu[e];
      mat[(size_t)T + s] = (R)md->lambda[e];
      mat[2 * (size_t)T + s] = (R)(md->alpha1 ? md->alpha1[e] : 0.0);
    }
  }

  CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CHECK(d_vid.ensure(sizeof(int4) * T));
  CHECK(d_dminv.ensure(sizeof(R) * 9 * (size_t)T));
  CHECK(d_vol.ensure(sizeof(R) * T));
  CHECK(d_mat.ensure(sizeof(R) * stride * (size_t)T));
  CHECK(d_lambda.ensure(sizeof(R) * 6 * (size_t)T));
  CHECK(d_pos.ensure(sizeof(R4<R>) * N));
  CHECK(d_oldp.ensure(sizeof(R4<R>) * N));
  CHECK(d_xprev.ensure(sizeof(R4<R>) * N));
  CHECK(d_resv.ensure(sizeof(R4<R>) * N));
  CHECK(d_vmass.ensure(sizeof(double) * N));
  CHECK(d_mass3.ensure(sizeof(double) * 3 * (size_t)N));
  CHECK(d_ri.ensure(sizeof(double4) * N));
  CHECK(d_s2e.ensure(sizeof(int) * T));
  CHECK(d_partials.ensure(sizeof(double) * 1024));
  CHECK(d_scalar.ensure(sizeof(double) * 8));  // [0] residual, [1] norm of resv, [7] k_residual_monitor's ticket
  CU(cudaMemsetAsync(d_scalar.p, 0, sizeof(double) * 8, stream));
  CHECK(h_scalar.ensure(sizeof(double) * 8));
  CHECK(d_gsync.ensure(sizeof(unsigned int) * 4));
  CHECK(h_gsync.ensure(sizeof(int) * 4));
  CU(cudaMemsetAsync(d_gsync.p, 0, sizeof(unsigned int) * 4, stream));
  {
    const char* e = std::getenv("MLXPBD_PERSISTENT");
    persistent = e && std::string(e) == "1";
    const char* q = std::getenv("MLXPBD_PDL");
    pdl = !(q && std::string(q) == "0");
    const char* hgv = std::getenv("MLXPBD_HOST_GRAPH");
    host_graph_on = !(hgv && std::string(hgv) == "0");
    const char* n = std::getenv("MLXPBD_PERSIST_CTAS");
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    persist_ctas = n ? std::max(1, std::min(std::atoi(n), sms)) : sms;
  }
  CHECK(d_pin_dofs.ensure(sizeof(int) * std::max<size_t>(pinned.size(), 1)));
  CHECK(d_pinx.ensure(sizeof(R) * std::max<size_t>(pinned.size(), 1)));
  CU(cudaMemcpyAsync(d_vid.p, vid.data(), sizeof(int4) * T, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_dminv.p, dminv.data(), sizeof(R) * 9 * (size_t)T, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_vol.p, vol.data(), sizeof(R) * T, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_mat.p, mat.data(), sizeof(R) * stride * (size_t)T, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_vmass.p, vmass_h.data(), sizeof(double) * N, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_mass3.p, mass3.data(), sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_s2e.p, s2e.data(), sizeof(int) * T, cudaMemcpyHostToDevice, stream));
  if (!pinned.empty())
    CU(cudaMemcpyAsync(d_pin_dofs.p, pinned.data(), sizeof(int) * pinned.size(), cudaMemcpyHostToDevice, stream));
  vid_sorted = vid;
  if (cluster_ok) vowner = mp.vowner;
  CHECK(plan_groups(md));
  if (md->mu && md->lambda) {
    pcg_G.resize(9 * (size_t)T);
    pcg_vol.resize(T);
    pcg_lame.resize(2 * (size_t)T);
    for (int sidx = 0; sidx < T; ++sidx) {
      const int e = s2e[sidx];
      for (int j = 0; j < 9; ++j) pcg_G[9 * (size_t)sidx + j] = md->DmInv[9 * (size_t)e + j];
      pcg_vol[sidx] = md->volume[e];
      pcg_lame[2 * (size_t)sidx] = md->mu[e];
      pcg_lame[2 * (size_t)sidx + 1] = md->lambda[e];
    }
  }
  CU(cudaStreamSynchronize(stream));
  return MLX_OK;
}

template <typename R>
static const void* cluster_kernel(int mat_kind, bool damp) {
  switch (mat_kind) {
    case MAT_NH: return (const void*)k_layer_cluster<R, MAT_NH, false>;
    case MAT_STVK_BLOCKS:
      return damp ? (const void*)k_layer_cluster<R, MAT_STVK_BLOCKS, true>
                  : (const void*)k_layer_cluster<R, MAT_STVK_BLOCKS, false>;
    default:
      return damp ? (const void*)k_layer_cluster<R, MAT_STVK_LAME, true>
                  : (const void*)k_layer_cluster<R, MAT_STVK_LAME, false>;
  }
}

// Chooses the cluster size: enough CTAs for ~64 tets of the largest colour
// each (at most 16), fewer if the device cannot co-schedule that cluster.
// The cluster path is left off when the vertex records of a part do not fit
// in a CTA's shared memory.
template <typename R>
int Solver<R>::plan_cluster(const mlx_mesh_desc* md, MeshPartition& mp) {
  cluster_ok = false;
  const char* env = std::getenv("MLXPBD_CLUSTER");
  if (!(env && std::string(env) == "1")) return MLX_OK;
  int maxc = 0;
  for (int c = 0; c < C; ++c) maxc = std::max(maxc, color_off[c + 1] - color_off[c]);
  int want = 1;
  while (want < 16 && want * 64 < maxc) want *= 2;
  if (const char* f = std::getenv("MLXPBD_CLUSTER_SIZE")) {
    int v = std::atoi(f);
    want = 1;
    while (want * 2 <= std::min(std::max(v, 1), 16)) want *= 2;
  }
  int optin = 0;
  CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  const void* fn = cluster_kernel<R>(mat_kind, damp);
  cudaFuncAttributes fa;
  CU(cudaFuncGetAttributes(&fa, fn));
  const long long budget = (long long)optin - (long long)fa.sharedSizeBytes - 1024;
  if (budget <= 0) return MLX_OK;
  CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
  cl_budget = budget;
  CU(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  const int nl = mat_kind == MAT_NH ? 2 : 6;
  for (int cs = want; cs >= 1; cs /= 2) {
    partition_mesh(N, T, md->t, cs, mp);
    const long long rec_bytes = (long long)mp.max_owned * (long long)sizeof(R4<R>);
    if (rec_bytes > budget) break;  // fewer CTAs would need even more shared memory
    std::vector<int> pc((size_t)C * cs, 0), tp(cs, 0);
    for (int e = 0; e < T; ++e) {
      ++pc[(size_t)(md->element_color[e] - 1) * cs + mp.tpart[e]];
      ++tp[mp.tpart[e]];
    }
    int maxr = 0, tmax = 0;
    for (int x : pc) maxr = std::max(maxr, x);
    for (int x : tp) tmax = std::max(tmax, x);
    // the multipliers of a CTA's tets join the records when they fit
    const long long lam_bytes = (long long)tmax * nl * (long long)sizeof(R);
    const bool lam_in_smem = rec_bytes + lam_bytes <= budget;
    const long long smem = rec_bytes + (lam_in_smem ? lam_bytes : 0);
    const int threads = std::min(std::max((maxr + 31) / 32 * 32, 64), kClusterMaxThreads);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cudaLaunchAttribute a;
    a.id = cudaLaunchAttributeClusterDimension;
    a.val.clusterDim.x = cs;
    a.val.clusterDim.y = 1;
    a.val.clusterDim.z = 1;
    cfg.attrs = &a;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (nclusters < 1) continue;
    cluster_ok = true;
    cl_size = cs;
    cl_threads = threads;
    cl_rec_slots = mp.max_owned;
    cl_lam_slots = lam_in_smem ? tmax : 0;
    cl_smem = (size_t)smem;
    return MLX_OK;
  }
  return MLX_OK;
}

template <typename R, int CM>
static const void* group_kernel_mode(int mat_kind, bool damp) {
  switch (mat_kind) {
    case MAT_NH:
      return (const void*)k_layer_groups<R, MAT_NH, false, CM>;
    case MAT_STVK_BLOCKS:
      return damp ? (const void*)k_layer_groups<R, MAT_STVK_BLOCKS, true, CM>
                  : (const void*)k_layer_groups<R, MAT_STVK_BLOCKS, false, CM>;
    default:
      return damp ? (const void*)k_layer_groups<R, MAT_STVK_LAME, true, CM>
                  : (const void*)k_layer_groups<R, MAT_STVK_LAME, false, CM>;
  }
}

// The group kernel of a material; mode as k_layer_groups' CMODE.
template <typename R>
static const void* group_kernel(int mat_kind, bool damp, int mode = 0) {
  if (mode == 1) return group_kernel_mode<R, 1>(mat_kind, damp);
  if (mode == 2) return group_kernel_mode<R, 2>(mat_kind, damp);
  return group_kernel_mode<R, 0>(mat_kind, damp);
}

// Groups of consecutive vertex-disconnected components for the
// component-group path: components must be ascending, contiguous vertex and
// element ranges (a merged batch is).  A colour phase of a group costs about
// one dependent chain of a tet projection (~2 us) per pass of the CTA over
// the group's tets of that colour, so groups take components in order while
// every colour still fits in one pass (and the records in shared memory); a
// larger component stands alone.  The path is taken when the slowest group's
// sweep is estimated shorter than the colour launches' (one dependent launch
// per colour, ~2.6 us, plus the colour's bytes at ~6.5 TB/s).
template <typename R>
static const void* cgroup_kernel(int mat_kind, bool damp) {
  switch (mat_kind) {
    case MAT_NH:
      return (const void*)k_layer_cgroups<R, MAT_NH, false>;
    case MAT_STVK_BLOCKS:
      return damp ? (const void*)k_layer_cgroups<R, MAT_STVK_BLOCKS, true>
                  : (const void*)k_layer_cgroups<R, MAT_STVK_BLOCKS, false>;
    default:
      return damp ? (const void*)k_layer_cgroups<R, MAT_STVK_LAME, true>
                  : (const void*)k_layer_cgroups<R, MAT_STVK_LAME, false>;
  }
}

template <typename R>
int Solver<R>::plan_groups(const mlx_mesh_desc* md) {
  groups_ok = false;
  const char* env = std::getenv("MLXPBD_GROUPS");
  const bool off = env && std::string(env) == "0", force = env && std::string(env) == "1";
  if (off || cluster_ok || persistent || T == 0) return MLX_OK;
  // components (union-find over the tets' corners)
  std::vector<int> parent(N);
  for (int v = 0; v < N; ++v) parent[v] = v;
  auto find = [&](int v) {
    while (parent[v] != v) {
      parent[v] = parent[parent[v]];
      v = parent[v];
    }
    return v;
  };
  for (int e = 0; e < T; ++e) {
    const int a = find(md->t[e] - 1);
    for (int k = 1; k < 4; ++k) {
      const int b = find(md->t[e + (size_t)k * T] - 1);
      if (a != b) parent[std::max(a, b)] = std::min(a, b);
    }
  }
  // component index of each vertex in order of first appearance; contiguous
  // vertex ranges means the index never decreases along the vertices
  std::vector<int> vcomp(N), cv0;
  {
    std::vector<int> label(N, -1);
    for (int v = 0; v < N; ++v) {
      const int r = find(v);
      if (label[r] < 0) {
        label[r] = (int)cv0.size();
        cv0.push_back(v);
      }
      vcomp[v] = label[r];
      if (v > 0 && vcomp[v] < vcomp[v - 1]) return MLX_OK;
    }
  }
  const int ncomp = (int)cv0.size();
  cv0.push_back(N);
  // tets of every (component, colour)
  std::vector<int> ccol((size_t)ncomp * C, 0), colcount(C, 0);
  int lastc = 0;
  for (int e = 0; e < T; ++e) {
    const int c = vcomp[md->t[e] - 1];
    if (c < lastc) return MLX_OK;  // elements are not grouped by component
    lastc = c;
    ++ccol[(size_t)c * C + md->element_color[e] - 1];
    ++colcount[md->element_color[e] - 1];
  }
  int optin = 0, sms = 0;
  CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  // Groups for cs CTAs each (cs = 1: one CTA; cs > 1: a thread-block cluster
  // whose CTAs hold contiguous spans of the group's vertex records).  A group
  // takes components while every colour still fits one pass of its cs CTAs
  // and closes once it holds cs * T / SMs tets, so many small components
  // spread over all SMs.  Returns the estimated sweep (us), or < 0.
  struct Plan {
    std::vector<int> gv0;
    long long max_span = 0;
    double t = -1;
  };
  auto form = [&](int cs, Plan& pl) -> double {
    const void* fn = cs == 1 ? group_kernel<R>(mat_kind, damp) : cgroup_kernel<R>(mat_kind, damp);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) { cudaGetLastError(); return -1; }
    const long long budget = (long long)optin - (long long)fa.sharedSizeBytes - 1024;
    const long long vmax = budget / (long long)sizeof(R4<R>) * cs;  // records of one group
    const long long cap = (long long)cs * kGroupThreads;
    std::vector<int> gv0{0}, acc(C, 0);
    long long gv = 0, max_gv = 0, max_passes = 0, gt = 0, max_span = 0;
    const long long target = ((long long)T * cs + sms - 1) / sms;
    auto passes = [&]() {
      long long n = 0;
      for (int q = 0; q < C; ++q) n += (acc[q] + cap - 1) / cap;
      return n;
    };
    auto close = [&]() {
      max_gv = std::max(max_gv, gv);
      max_span = std::max(max_span, (gv + cs - 1) / cs);
      max_passes = std::max(max_passes, passes());
    };
    for (int c = 0; c < ncomp; ++c) {
      const long long nv = cv0[c + 1] - cv0[c];
      if (nv > vmax) return -1;
      bool fits = gv + nv <= vmax;
      for (int q = 0; q < C && fits; ++q) fits = acc[q] + ccol[(size_t)c * C + q] <= cap;
      if (gv > 0 && (!fits || gt >= target)) {
        gv0.push_back(cv0[c]);
        close();
        std::fill(acc.begin(), acc.end(), 0);
        gv = 0;
        gt = 0;
      }
      for (int q = 0; q < C; ++q) {
        acc[q] += ccol[(size_t)c * C + q];
        gt += ccol[(size_t)c * C + q];
      }
      gv += nv;
    }
    gv0.push_back(N);
    close();
    const long long G = (long long)gv0.size() - 1;
    long long resident = sms;  // groups in flight at once
    double per_phase = 2.0;    // us: the dependent chain of one projection
    if (cs > 1) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(cs * std::min<long long>(G, 1 << 16)));
      cfg.blockDim = dim3(kGroupThreads);
      cfg.dynamicSmemBytes = (size_t)max_span * sizeof(R4<R>);
      cudaLaunchAttribute a;
      a.id = cudaLaunchAttributeClusterDimension;
      a.val.clusterDim.x = cs;
      a.val.clusterDim.y = 1;
      a.val.clusterDim.z = 1;
      cfg.attrs = &a;
      cfg.numAttrs = 1;
      int ncl = 0;
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)std::max<size_t>(cfg.dynamicSmemBytes, 16)) != cudaSuccess ||
          cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg) != cudaSuccess || ncl < 1) {
        cudaGetLastError();
        return -1;
      }
      resident = ncl;
      // measured on B200 (config 3 and 16,384 cantilevers): the cluster
      // barrier after remote stores and the distributed-shared-memory
      // gathers put a phase well above a colour launch
      per_phase = 6.0;
    }
    pl.gv0 = gv0;
    pl.max_span = max_span;
    pl.t = per_phase * (double)max_passes * (double)((G + resident - 1) / resident);
    return pl.t;
  };
  double t_colours = 0;
  for (int q = 0; q < C; ++q)
    if (colcount[q]) t_colours += 2.6 + (double)colcount[q] * (double)bytes_per_tet() / 6.5e6;
  int cs_force = 0;
  if (const char* f = std::getenv("MLXPBD_GROUP_CS")) cs_force = std::atoi(f);
  Plan best;
  int best_cs = 0;
  for (int cs : {1, 2, 4, 8}) {
    if (cs_force > 0 && cs != cs_force) continue;
    Plan pl;
    const double t = form(cs, pl);
    if (t < 0) continue;
    if (best_cs == 0 || t < best.t) {
      best = pl;
      best_cs = cs;
    }
  }
  if (best_cs == 0) return MLX_OK;
  if (!force && cs_force <= 0 && best.t >= t_colours) return MLX_OK;
  const std::vector<int>& gv0 = best.gv0;
  const int G = (int)gv0.size() - 1;
  const int cs = best_cs;
  // each group's pins must be one range of the pinned list, in group order
  // (true when the list is ascending); a group applies its range in order
  std::vector<int> gpin(G + 1, 0);
  {
    int lastg = 0;
    for (size_t i = 0; i < pinned.size(); ++i) {
      const int g = (int)(std::upper_bound(gv0.begin(), gv0.end(), pinned[i] / 3) - gv0.begin()) - 1;
      if (g < lastg) return MLX_OK;
      lastg = g;
      ++gpin[g + 1];
    }
    for (int q = 0; q < G; ++q) gpin[q + 1] += gpin[q];
  }
  // group of every tet (sorted order) and its corner slots (cs = 1: vertex -
  // v0; cs > 1: rank << 24 | slot in that rank's span of ceil(nv / cs))
  tgroup_sorted.assign(T, 0);
  std::vector<int4> tloc(T);
  for (int sidx = 0; sidx < T; ++sidx) {
    const int4 v = vid_sorted[sidx];
    const int g = (int)(std::upper_bound(gv0.begin(), gv0.end(), v.x) - gv0.begin()) - 1;
    tgroup_sorted[sidx] = g;
    const int b = gv0[g];
    if (cs == 1) {
      tloc[sidx] = make_int4(v.x - b, v.y - b, v.z - b, v.w - b);
    } else {
      const int span = (gv0[g + 1] - b + cs - 1) / cs;
      auto code = [&](int u) { return (((u - b) / span) << 24) | ((u - b) % span); };
      tloc[sidx] = make_int4(code(v.x), code(v.y), code(v.z), code(v.w));
    }
  }
  gr_smem = (size_t)best.max_span * sizeof(R4<R>);
  if (cs == 1) {
    CU(cudaFuncSetAttribute(group_kernel<R>(mat_kind, damp), cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)std::max<size_t>(gr_smem, 16)));
    for (int mode = 1; mode <= 2; ++mode)
      CU(cudaFuncSetAttribute(group_kernel<R>(mat_kind, damp, mode), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)std::max<size_t>(gr_smem, 16)));
  } else {
    CU(cudaFuncSetAttribute(cgroup_kernel<R>(mat_kind, damp), cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)std::max<size_t>(gr_smem, 16)));
  }
  CHECK(d_gv0.ensure(sizeof(int) * gv0.size()));
  CHECK(d_tloc.ensure(sizeof(int4) * (size_t)T));
  CHECK(d_gpin.ensure(sizeof(int) * gpin.size()));
  CU(cudaMemcpyAsync(d_gv0.p, gv0.data(), sizeof(int) * gv0.size(), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_tloc.p, tloc.data(), sizeof(int4) * (size_t)T, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_gpin.p, gpin.data(), sizeof(int) * gpin.size(), cudaMemcpyHostToDevice, stream));
  CU(cudaStreamSynchronize(stream));
  gr_G = G;
  gr_cs = cs;
  groups_ok = true;
  return MLX_OK;
}

// k_layer_groups<R, material, damping, CM> on a launch configuration.
template <typename R, int CM>
static cudaError_t launch_group_kernel(cudaLaunchConfig_t* cfg, int mat_kind, bool damp, TetData<R> td, GroupArgs ga,
                                       R4<R>* p, const R4<R>* oldp, R inv_h2, R inv_h, const DevContacts& dc,
                                       double h, double cr, const R* pv, const HostContactGroups& hc) {
  switch (mat_kind) {
    case MAT_NH:
      return cudaLaunchKernelEx(cfg, k_layer_groups<R, MAT_NH, false, CM>, td, ga, p, oldp, inv_h2, inv_h, dc, oldp, h,
                                cr, pv, hc);
    case MAT_STVK_BLOCKS:
      return damp ? cudaLaunchKernelEx(cfg, k_layer_groups<R, MAT_STVK_BLOCKS, true, CM>, td, ga, p, oldp, inv_h2,
                                       inv_h, dc, oldp, h, cr, pv, hc)
                  : cudaLaunchKernelEx(cfg, k_layer_groups<R, MAT_STVK_BLOCKS, false, CM>, td, ga, p, oldp, inv_h2,
                                       inv_h, dc, oldp, h, cr, pv, hc);
    default:
      return damp ? cudaLaunchKernelEx(cfg, k_layer_groups<R, MAT_STVK_LAME, true, CM>, td, ga, p, oldp, inv_h2,
                                       inv_h, dc, oldp, h, cr, pv, hc)
                  : cudaLaunchKernelEx(cfg, k_layer_groups<R, MAT_STVK_LAME, false, CM>, td, ga, p, oldp, inv_h2,
                                       inv_h, dc, oldp, h, cr, pv, hc);
  }
}

template <typename R>
int Solver<R>::launch_groups(const LayerStatic& ls, const int* dint, const mlx_solve_params* P, int iterations,
                             const DevContacts& dc, const HostContactGroups* hc) {
  GroupArgs ga;
  ga.list = ls.identity_list ? nullptr : dint + ls.o_list;
  ga.off = dint + ls.o_goff;
  ga.gv0 = d_gv0.as<int>();
  ga.tloc = d_tloc.as<int4>();
  ga.pin_off = d_gpin.as<int>();
  ga.pin_dofs = d_pin_dofs.as<int>();
  ga.C = C;
  ga.G = gr_G;
  ga.iterations = iterations;
  ga.one_per_thread = ls.gr_one;
  const R hR = (R)P->h;
  const R inv_h2 = R(1) / (hR * hR), inv_h = R(1) / hR;
  TetData<R> td = tets();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(gr_G);
  cfg.blockDim = dim3(kGroupThreads);
  cfg.dynamicSmemBytes = gr_smem;
  cfg.stream = stream;
  const R4<R>* oldp = d_oldp.as<R4<R>>();
  const R* pv = d_pinx.as<R>();
  const double h = P->h, cr = P->contact_resistance;
  if (gr_cs > 1) {
    // a cluster of gr_cs CTAs per group (no contact phase on this path)
    cfg.gridDim = dim3(gr_G * gr_cs);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = gr_cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    switch (mat_kind) {
      case MAT_NH:
        e = cudaLaunchKernelEx(&cfg, k_layer_cgroups<R, MAT_NH, false>, td, ga, pos(), oldp, inv_h2, inv_h, pv);
        break;
      case MAT_STVK_BLOCKS:
        e = damp ? cudaLaunchKernelEx(&cfg, k_layer_cgroups<R, MAT_STVK_BLOCKS, true>, td, ga, pos(), oldp, inv_h2,
                                      inv_h, pv)
                 : cudaLaunchKernelEx(&cfg, k_layer_cgroups<R, MAT_STVK_BLOCKS, false>, td, ga, pos(), oldp, inv_h2,
                                      inv_h, pv);
        break;
      default:
        e = damp ? cudaLaunchKernelEx(&cfg, k_layer_cgroups<R, MAT_STVK_LAME, true>, td, ga, pos(), oldp, inv_h2,
                                      inv_h, pv)
                 : cudaLaunchKernelEx(&cfg, k_layer_cgroups<R, MAT_STVK_LAME, false>, td, ga, pos(), oldp, inv_h2,
                                      inv_h, pv);
    }
    if (e != cudaSuccess)
      return set_error(MLX_ERR_CUDA, std::string("cluster group layer launch: ") + cudaGetErrorString(e));
    return MLX_OK;
  }
  HostContactGroups none{};
  const HostContactGroups& hg_ = hc ? *hc : none;
  const cudaError_t e =
      dc.colored ? launch_group_kernel<R, 1>(&cfg, mat_kind, damp, td, ga, pos(), oldp, inv_h2, inv_h, dc, h, cr, pv, hg_)
      : hc       ? launch_group_kernel<R, 2>(&cfg, mat_kind, damp, td, ga, pos(), oldp, inv_h2, inv_h, dc, h, cr, pv, hg_)
                 : launch_group_kernel<R, 0>(&cfg, mat_kind, damp, td, ga, pos(), oldp, inv_h2, inv_h, dc, h, cr, pv, hg_);
  if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("group layer launch: ") + cudaGetErrorString(e));
  return MLX_OK;
}

// Diagnostic of the grid barrier's bounded wait: thread 0 waits for a count
// nothing increments, so the wait runs out after limit_ns.
__global__ void k_probe_grid_wait(unsigned* count, int* error, unsigned long long limit_ns, int* timed_out) {
  if (threadIdx.x == 0) *timed_out = wait_count_ge(count, 1u, error, limit_ns) ? 0 : 1;
}

__global__ void k_iota(int* __restrict__ a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}
__global__ void k_last_count(const int* __restrict__ scan, const int* __restrict__ flag, int T, int* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = T > 0 ? scan[T - 1] + flag[T - 1] : 0;
}

template <typename R>
int Solver<R>::build_layers(const double* p, const double* oldp, double h, int ordering, const int32_t* order,
                            const double* dminv, const double* sorted_layers, int L, const uint8_t* forced,
                            int32_t* sets, int32_t* num_rigids, uint8_t* is_elastic, uint8_t* is_boundary,
                            uint8_t* is_rigid_vertex, int32_t* vertex_body) {
  if (!sorted_layers || !forced || !sets || !num_rigids || L < 1)
    return set_error(MLX_ERR_ARGUMENT, "bad layer-builder arguments");
  if (ordering == 0 && (!p || !oldp || !dminv || !(h > 0)))
    return set_error(MLX_ERR_ARGUMENT, "strain-rate ordering needs p, oldp, DmInv and h > 0");
  if (ordering == 1 && !order) return set_error(MLX_ERR_ARGUMENT, "ordering 1 needs the order");
  if (ordering != 0 && ordering != 1) return set_error(MLX_ERR_ARGUMENT, "ordering must be 0 or 1");
  for (int l = 1; l < L; ++l)
    if (sorted_layers[l] < sorted_layers[l - 1]) return set_error(MLX_ERR_ARGUMENT, "layers must be ascending");
  if (T == 0 || N == 0) {
    for (int l = 0; l < L; ++l) num_rigids[l] = 0;
    return MLX_OK;
  }
  DeviceGuard g(device);
  const int bs = 256, tb = blocks_for(T, bs), nbk = blocks_for(N, bs);
  CHECK(lb_order.ensure(sizeof(int) * std::max(T, 1)));
  CHECK(lb_rank.ensure(sizeof(int) * std::max(T, 1)));
  CHECK(lb_forced.ensure(std::max(T, 1)));
  CHECK(lb_parent.ensure(sizeof(int) * std::max(T, 1)));
  CHECK(lb_root.ensure(sizeof(int) * std::max(T, 1)));
  CHECK(lb_flag.ensure(sizeof(int) * std::max(T, 1)));
  CHECK(lb_scan.ensure(sizeof(int) * std::max(T, 1)));
  CHECK(lb_sets.ensure(sizeof(int32_t) * std::max<size_t>((size_t)T * L, 1)));
  CHECK(lb_isE.ensure(std::max<size_t>((size_t)T * L, 1)));
  CHECK(lb_rep.ensure(sizeof(int) * std::max(N, 1)));
  CHECK(lb_key.ensure(sizeof(int) * std::max(N, 1)));
  CHECK(lb_touch.ensure(sizeof(int) * std::max(N, 1)));
  CHECK(lb_isBV.ensure(std::max<size_t>((size_t)N * L, 1)));
  CHECK(lb_isRV.ensure(std::max<size_t>((size_t)N * L, 1)));
  CHECK(lb_body.ensure(sizeof(int32_t) * std::max<size_t>((size_t)N * L, 1)));
  CHECK(lb_small.ensure(sizeof(int) * (size_t)(L + 1)));
  int* err = lb_small.as<int>() + L;
  CU(cudaMemsetAsync(lb_small.p, 0, sizeof(int) * (size_t)(L + 1), stream));
  CU(cudaMemcpyAsync(lb_forced.p, forced, T, cudaMemcpyHostToDevice, stream));
  const int4* vid = d_vid.as<int4>();
  const int* s2e_d = d_s2e.as<int>();
  // ---- the order ----
  if (ordering == 0) {
    CHECK(lb_p.ensure(sizeof(double) * 3 * (size_t)N));
    CHECK(lb_oldp.ensure(sizeof(double) * 3 * (size_t)N));
    CHECK(lb_norms.ensure(sizeof(double) * std::max(T, 1)));
    CHECK(lb_norms_sorted.ensure(sizeof(double) * std::max(T, 1)));
    CHECK(lb_elems.ensure(sizeof(int) * std::max(T, 1)));
    if (dminv != lb_dminv_src || !lb_dminv.p) {
      CHECK(lb_dminv.ensure(sizeof(double) * 9 * (size_t)T));
      CU(cudaMemcpyAsync(lb_dminv.p, dminv, sizeof(double) * 9 * (size_t)T, cudaMemcpyHostToDevice, stream));
      lb_dminv_src = dminv;
    }
    CU(cudaMemcpyAsync(lb_p.p, p, sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(lb_oldp.p, oldp, sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice, stream));
    const double inv_h2 = 1.0 / (h * h);
    k_strain_rate_norms<<<tb, bs, 0, stream>>>(vid, s2e_d, T, lb_dminv.as<double>(), lb_p.as<double>(),
                                               lb_oldp.as<double>(), inv_h2, lb_norms.as<double>(),
                                               lb_elems.as<int>());
    CU(cudaGetLastError());
    // stable ascending sort of (measure, element): the order of sort(...,"ascend")
    size_t tmp = 0;
    CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, lb_norms.as<double>(), lb_norms_sorted.as<double>(),
                                       lb_elems.as<int>(), lb_order.as<int>(), T, 0, 64, stream));
    CHECK(lb_tmp.ensure(std::max<size_t>(tmp, 16)));
    CU(cub::DeviceRadixSort::SortPairs(lb_tmp.p, tmp, lb_norms.as<double>(), lb_norms_sorted.as<double>(),
                                       lb_elems.as<int>(), lb_order.as<int>(), T, 0, 64, stream));
  } else {
    std::vector<int> o(T);
    for (int q = 0; q < T; ++q) {
      o[q] = order[q] - 1;
      if (o[q] < 0 || o[q] >= T) return set_error(MLX_ERR_ARGUMENT, "order entry out of range");
    }
    CU(cudaMemcpyAsync(lb_order.p, o.data(), sizeof(int) * (size_t)T, cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));  // o is a pageable host source
  }
  k_order_rank<<<tb, bs, 0, stream>>>(lb_order.as<int>(), T, lb_rank.as<int>());
  CU(cudaGetLastError());
  size_t stmp = 0;
  CU(cub::DeviceScan::ExclusiveSum(nullptr, stmp, lb_flag.as<int>(), lb_scan.as<int>(), T, stream));
  if (lb_tmp.bytes < stmp) CHECK(lb_tmp.ensure(stmp));
  // ---- every layer ----
  for (int l = 0; l < L; ++l) {
    const int end = std::min((int)std::floor((sorted_layers[l] / 100.0) * T), T);
    int32_t* sl = lb_sets.as<int32_t>() + (size_t)T * l;
    CU(cudaMemsetAsync(lb_rep.p, 0x7f, sizeof(int) * (size_t)N, stream));
    k_uf_init<<<tb, bs, 0, stream>>>(lb_rank.as<int>(), lb_forced.as<uint8_t>(), T, end, lb_parent.as<int>());
    k_uf_rep<<<tb, bs, 0, stream>>>(vid, s2e_d, T, lb_parent.as<int>(), lb_rep.as<int>());
    k_uf_unite<<<tb, bs, 0, stream>>>(vid, s2e_d, T, lb_parent.as<int>(), lb_rep.as<int>(), err);
    k_uf_roots<<<tb, bs, 0, stream>>>(T, lb_parent.as<int>(), lb_root.as<int>(), lb_flag.as<int>(), err);
    CU(cudaGetLastError());
    size_t st2 = lb_tmp.bytes;
    CU(cub::DeviceScan::ExclusiveSum(lb_tmp.p, st2, lb_flag.as<int>(), lb_scan.as<int>(), T, stream));
    k_uf_label<<<tb, bs, 0, stream>>>(T, lb_root.as<int>(), lb_scan.as<int>(), sl);
    k_last_count<<<1, 32, 0, stream>>>(lb_scan.as<int>(), lb_flag.as<int>(), T, lb_small.as<int>() + l);
    // findBoundaryVertices of this layer
    CU(cudaMemsetAsync(lb_key.p, 0xff, sizeof(int) * (size_t)N, stream));
    CU(cudaMemsetAsync(lb_touch.p, 0, sizeof(int) * (size_t)N, stream));
    k_bv_keys<<<tb, bs, 0, stream>>>(vid, s2e_d, T, sl, lb_key.as<int>(), lb_touch.as<int>());
    k_bv_masks<<<nbk, bs, 0, stream>>>(N, T, sl, lb_key.as<int>(), lb_touch.as<int>(),
                                       lb_isBV.as<uint8_t>() + (size_t)N * l, lb_isRV.as<uint8_t>() + (size_t)N * l,
                                       lb_body.as<int32_t>() + (size_t)N * l);
    k_elastic_mask<<<tb, bs, 0, stream>>>(T, sl, lb_isE.as<uint8_t>() + (size_t)T * l);
    CU(cudaGetLastError());
  }
  std::vector<int> small(L + 1);
  CU(cudaMemcpyAsync(small.data(), lb_small.p, sizeof(int) * (size_t)(L + 1), cudaMemcpyDeviceToHost, stream));
  CU(cudaMemcpyAsync(sets, lb_sets.p, sizeof(int32_t) * (size_t)T * L, cudaMemcpyDeviceToHost, stream));
  if (is_elastic) CU(cudaMemcpyAsync(is_elastic, lb_isE.p, (size_t)T * L, cudaMemcpyDeviceToHost, stream));
  if (is_boundary) CU(cudaMemcpyAsync(is_boundary, lb_isBV.p, (size_t)N * L, cudaMemcpyDeviceToHost, stream));
  if (is_rigid_vertex) CU(cudaMemcpyAsync(is_rigid_vertex, lb_isRV.p, (size_t)N * L, cudaMemcpyDeviceToHost, stream));
  if (vertex_body)
    CU(cudaMemcpyAsync(vertex_body, lb_body.p, sizeof(int32_t) * (size_t)N * L, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  if (small[L]) return set_error(MLX_ERR_LIMIT, "union-find step bound reached");
  for (int l = 0; l < L; ++l) num_rigids[l] = small[l];
  return MLX_OK;
}

// Whether every layer of `ld` finds its static data cached in `w` unchanged
// (the check build_static makes, plus the rigid-element count).
template <typename R>
bool Solver<R>::statics_hit(const mlx_layer_desc* ld, const LayerWork& w) const {
  for (int layer = 0; layer < ld->num_layers; ++layer) {
    const int col = ld->layers_map[layer] - 1;
    if (col < 0 || col >= (int)w.cache.size() || !w.cache[col]) return false;
    const LayerStatic& ls = *w.cache[col];
    const uint8_t* isE = ld->is_elastic_element + (size_t)T * col;
    const uint8_t* isR = ld->is_rigid_element + (size_t)T * col;
    const int32_t* rid = ld->vertex_rigid_body + (size_t)N * col;
    const uint8_t* isBV = ld->is_boundary_vertex + (size_t)N * col;
    const uint8_t* isRV = ld->is_rigid_vertex + (size_t)N * col;
    if (!(ls.valid && ls.nb == ld->num_rigids[col] && std::memcmp(ls.isE.data(), isE, T) == 0 &&
          std::memcmp(ls.isBV.data(), isBV, N) == 0 && std::memcmp(ls.isRV.data(), isRV, N) == 0 &&
          std::memcmp(ls.rid.data(), rid, sizeof(int32_t) * N) == 0))
      return false;
    int nre = 0;
    for (int e = 0; e < T; ++e) nre += isR[e] != 0;
    if (nre != ls.n_rigid_elements) return false;
  }
  return true;
}

template <typename R>
int Solver<R>::build_static(const mlx_layer_desc* ld, int col, LayerStatic& ls, bool capturing) {
  const uint8_t* isE = ld->is_elastic_element + (size_t)T * col;
  const uint8_t* isR = ld->is_rigid_element + (size_t)T * col;
  const int32_t* rid = ld->vertex_rigid_body + (size_t)N * col;
  const uint8_t* isBV = ld->is_boundary_vertex + (size_t)N * col;
  const uint8_t* isRV = ld->is_rigid_vertex + (size_t)N * col;
  int nb = ld->num_rigids[col];
  if (ls.valid && ls.nb == nb && std::memcmp(ls.isE.data(), isE, T) == 0 &&
      std::memcmp(ls.isBV.data(), isBV, N) == 0 && std::memcmp(ls.isRV.data(), isRV, N) == 0 &&
      std::memcmp(ls.rid.data(), rid, sizeof(int32_t) * N) == 0) {
    int nre = 0;
    for (int e = 0; e < T; ++e) nre += isR[e] != 0;
    ls.n_rigid_elements = nre;
    ls.tile = col < (int)tiles.size() ? tiles[col] : std::vector<int>();
    return MLX_OK;
  }
  if (nb < 0) return set_error(MLX_ERR_ARGUMENT, "num_rigids < 0");
  if (capturing) return set_error(MLX_ERR_ARGUMENT, "layer cache miss inside a captured step");
  ls.valid = false;
  ls.tile = col < (int)tiles.size() ? tiles[col] : std::vector<int>();
  ls.isE.assign(isE, isE + T);
  ls.isBV.assign(isBV, isBV + N);
  ls.isRV.assign(isRV, isRV + N);
  ls.rid.assign(rid, rid + N);
  ls.nb = nb;
  int nre = 0;
  for (int e = 0; e < T; ++e) nre += isR[e] != 0;
  ls.n_rigid_elements = nre;
  // elastic tets per colour in sorted order
  std::vector<int> list;
  list.reserve(T);
  ls.color_count.assign(C, 0);
  ls.color_start.assign(C, 0);
  for (int c = 0; c < C; ++c) {
    ls.color_start[c] = (int)list.size();
    for (int s = color_off[c]; s < color_off[c + 1]; ++s)
      if (isE[s2e[s]]) list.push_back(s);
    ls.color_count[c] = (int)list.size() - ls.color_start[c];
  }
  ls.identity_list = (int)list.size() == T;
  // bodies
  std::vector<int> bvo(nb + 1, 0), bo(nb + 1, 0);
  for (int v = 0; v < N; ++v) {
    int b = rid[v];
    if (b < 0 || b > nb) return set_error(MLX_ERR_ARGUMENT, "vertex_rigid_body id out of [0, num_rigids]");
    if (b > 0) ++bvo[b];
    if (isBV[v]) {
      if (b == 0) return set_error(MLX_ERR_ARGUMENT, "a boundary vertex has no rigid body");
      ++bo[b];
    }
  }
  for (int b = 1; b <= nb; ++b) { bvo[b] += bvo[b - 1]; bo[b] += bo[b - 1]; }
  std::vector<int> bverts(bvo[nb]), bnd(bo[nb]);
  {
    std::vector<int> f1(bvo.begin(), bvo.end() - 1), f2(bo.begin(), bo.end() - 1);
    for (int v = 0; v < N; ++v) {
      int b = rid[v];
      if (b > 0) bverts[f1[b - 1]++] = v;
      if (isBV[v]) bnd[f2[b - 1]++] = v;
    }
  }
  ls.n_bnd = bo[nb];
  // pack
  ls.packed.clear();
  auto put = [&](const std::vector<int>& a) {
    size_t o = ls.packed.size();
    ls.packed.insert(ls.packed.end(), a.begin(), a.end());
    return o;
  };
  ls.o_bvo = put(bvo);
  ls.o_bv = put(bverts);
  ls.o_bo = put(bo);
  ls.o_bnd = put(bnd);
  ls.o_list = put(ls.identity_list ? std::vector<int>() : list);
  ls.o_vb = ls.packed.size();
  ls.packed.insert(ls.packed.end(), rid, rid + N);
  // colour ranges for the persistent kernel (starts index the list, or the
  // sorted order when the list is the identity)
  std::vector<int> cstart(C);
  for (int c = 0; c < C; ++c) cstart[c] = ls.identity_list ? color_off[c] : ls.color_start[c];
  ls.o_cstart = put(cstart);
  ls.o_ccount = put(ls.color_count);
  // CTAs of the per-body kernels: a body of more than kSmallBody vertices
  // alone, the others kItemInts per CTA (one warp each) in body order
  {
    std::vector<int> items, small;
    for (int b = 0; b < nb; ++b) {
      if (bvo[b + 1] - bvo[b] > kSmallBody) {
        items.push_back(b);
        items.push_back(kLargeItem);
        for (int q = 2; q < kItemInts; ++q) items.push_back(-1);
      } else {
        small.push_back(b);
      }
    }
    for (size_t i = 0; i < small.size(); i += kItemInts)
      for (int q = 0; q < kItemInts; ++q) items.push_back(i + q < small.size() ? small[i + q] : -1);
    ls.n_items = (int)(items.size() / kItemInts);
    ls.o_items = put(items);
  }
  // (colour, group) ranges of the elastic tets for the component-group path:
  // within a colour the elastic tets are in element order, so each group's
  // are one range when the groups are ascending element ranges
  ls.gr_ok = false;
  if (groups_ok) {
    const int G = gr_G;
    std::vector<int> goff((size_t)C * G + 1, 0);
    bool mono = true;
    int maxr = 0;
    for (int c = 0; c < C && mono; ++c) {
      const int b = ls.identity_list ? color_off[c] : ls.color_start[c];
      const int n = ls.color_count[c];
      int last = -1;
      for (int q = 0; q < n; ++q) {
        const int sidx = ls.identity_list ? b + q : list[b + q];
        const int g = tgroup_sorted[sidx];
        if (g < last) { mono = false; break; }
        last = g;
        ++goff[(size_t)c * G + g + 1];
      }
    }
    if (mono) {
      for (size_t q = 1; q < goff.size(); ++q) maxr = std::max(maxr, goff[q]);
      // counts -> starts (in list positions, or sorted ids for the identity)
      for (int c = 0; c < C; ++c) {
        int run = ls.identity_list ? color_off[c] : ls.color_start[c];
        for (int g = 0; g < G; ++g) {
          const int cnt = goff[(size_t)c * G + g + 1];
          goff[(size_t)c * G + g] = run;
          run += cnt;
        }
      }
      goff[(size_t)C * G] = ls.identity_list ? T : (int)list.size();
      ls.gr_one = maxr <= gr_cs * kGroupThreads ? 1 : 0;
      ls.o_goff = put(goff);
      ls.gr_ok = true;
    }
  }
  if (cluster_ok) {
    // the elastic list (or the identity) is in sorted order, which is
    // (colour, part) order on the cluster path
    const int P = cl_size;
    std::vector<int> off((size_t)C * P + 1, 0), cols;
    for (int c = 0; c < C; ++c)
      for (int s = color_off[c]; s < color_off[c + 1]; ++s)
        if (isE[s2e[s]]) ++off[(size_t)c * P + tpart_sorted[s] + 1];
    for (size_t q = 1; q < off.size(); ++q) off[q] += off[q - 1];
    int maxr = 0;
    for (int c = 0; c < C; ++c) {
      if (off[(size_t)(c + 1) * P] > off[(size_t)c * P]) cols.push_back(c);
      for (int r = 0; r < P; ++r) maxr = std::max(maxr, off[(size_t)c * P + r + 1] - off[(size_t)c * P + r]);
    }
    // shared-memory multiplier slots: a rank's tets in colour order
    std::vector<int> lb((size_t)C * P, 0);
    for (int r = 0; r < P; ++r) {
      int acc = 0;
      for (int c = 0; c < C; ++c) {
        lb[(size_t)c * P + r] = acc;
        acc += off[(size_t)c * P + r + 1] - off[(size_t)c * P + r];
      }
    }
    ls.cl_nC = (int)cols.size();
    ls.cl_max_range = maxr;
    ls.o_cloff = put(off);
    ls.o_clcol = put(cols);
    ls.o_cllb = put(lb);
    CHECK(build_cluster_slots(ls, list));
  }
  CHECK(ls.dev.ensure(sizeof(int) * ls.packed.size()));
  CHECK(ls.dev_rigid.ensure(N));
  CU(cudaMemcpyAsync(ls.dev.p, ls.packed.data(), sizeof(int) * ls.packed.size(), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(ls.dev_rigid.p, isRV, N, cudaMemcpyHostToDevice, stream));
  // the host copies above are pageable: make sure they finished before the
  // cached vectors can change
  CU(cudaStreamSynchronize(stream));
  ls.valid = true;
  return MLX_OK;
}

template <typename R>
int Solver<R>::launch_color(int c, const LayerStatic& ls, const int* dlist, R h, int bs_override,
                            const DevContacts* cc, const int* vert_body, double hd, double cr) {
  int count = ls.color_count[c];
  if (count == 0 && !cc) return MLX_OK;
  const int bs = bs_override > 0 ? bs_override : (ls.tile.empty() || ls.tile[c] <= 0 ? kDefaultTile : ls.tile[c]);
  R inv_h2 = R(1) / (h * h), inv_h = R(1) / h;
  TetData<R> td = tets();
  const int* list = ls.identity_list ? nullptr : dlist;
  int begin = ls.identity_list ? color_off[c] : ls.color_start[c];
  const R4<R>* oldp = d_oldp.as<R4<R>>();
  R4<R>* p = pos();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks_for(count, bs));
  cfg.blockDim = dim3(bs);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaError_t e;
  if (cc) {
    // contact_coloring: extra CTAs for the elastic contacts of this colour
    // phase (their number is known on the device only: a fixed grid strides)
    const int tb = blocks_for(count, bs);
    const int extra = std::max(1, std::min(32, blocks_for(N, bs) / std::max(C, 1) + 1));
    cfg.gridDim = dim3(tb + extra);
    const R4<R>* x0 = d_oldp.as<R4<R>>();
    switch (mat_kind) {
      case MAT_NH:
        e = cudaLaunchKernelEx(&cfg, k_project_color_cc<R, MAT_NH, false>, td, list, begin, count, p, oldp, inv_h2,
                               inv_h, tb, *cc, c, vert_body, x0, hd, cr);
        break;
      case MAT_STVK_BLOCKS:
        e = damp ? cudaLaunchKernelEx(&cfg, k_project_color_cc<R, MAT_STVK_BLOCKS, true>, td, list, begin, count, p,
                                      oldp, inv_h2, inv_h, tb, *cc, c, vert_body, x0, hd, cr)
                 : cudaLaunchKernelEx(&cfg, k_project_color_cc<R, MAT_STVK_BLOCKS, false>, td, list, begin, count, p,
                                      oldp, inv_h2, inv_h, tb, *cc, c, vert_body, x0, hd, cr);
        break;
      default:
        e = damp ? cudaLaunchKernelEx(&cfg, k_project_color_cc<R, MAT_STVK_LAME, true>, td, list, begin, count, p,
                                      oldp, inv_h2, inv_h, tb, *cc, c, vert_body, x0, hd, cr)
                 : cudaLaunchKernelEx(&cfg, k_project_color_cc<R, MAT_STVK_LAME, false>, td, list, begin, count, p,
                                      oldp, inv_h2, inv_h, tb, *cc, c, vert_body, x0, hd, cr);
    }
    if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("colour launch: ") + cudaGetErrorString(e));
    return MLX_OK;
  }
  switch (mat_kind) {
    case MAT_NH:
      e = cudaLaunchKernelEx(&cfg, k_project_color<R, MAT_NH, false>, td, list, begin, count, p, oldp, inv_h2, inv_h);
      break;
    case MAT_STVK_BLOCKS:
      e = damp ? cudaLaunchKernelEx(&cfg, k_project_color<R, MAT_STVK_BLOCKS, true>, td, list, begin, count, p, oldp,
                                    inv_h2, inv_h)
               : cudaLaunchKernelEx(&cfg, k_project_color<R, MAT_STVK_BLOCKS, false>, td, list, begin, count, p, oldp,
                                    inv_h2, inv_h);
      break;
    default:
      e = damp ? cudaLaunchKernelEx(&cfg, k_project_color<R, MAT_STVK_LAME, true>, td, list, begin, count, p, oldp,
                                    inv_h2, inv_h)
               : cudaLaunchKernelEx(&cfg, k_project_color<R, MAT_STVK_LAME, false>, td, list, begin, count, p, oldp,
                                    inv_h2, inv_h);
  }
  if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("colour launch: ") + cudaGetErrorString(e));
  return MLX_OK;
}

template <typename R>
int Solver<R>::residual(const ContactData& cd, double contact_resistance, double h, double* out,
                        const DevContacts* dc) {
  const int bs = 256;
  int tetBlocks = std::min(blocks_for(T, bs), 592);
  int cBlocks = cd.K > 0 ? std::min(blocks_for(cd.K, bs), 64) : 0;
  R inv_h2 = R(1) / ((R)h * (R)h), inv_h = R(1) / (R)h;
  double inv_h2_d = 1.0 / (h * h);
  TetData<R> td = tets();
  double* partials = d_partials.as<double>();
  switch (mat_kind) {
    case MAT_NH:
      k_residual_partials<R, MAT_NH><<<tetBlocks + cBlocks, bs, 0, stream>>>(td, pos(), cd, contact_resistance, inv_h2, inv_h, inv_h2_d, tetBlocks, partials);
      break;
    case MAT_STVK_BLOCKS:
      k_residual_partials<R, MAT_STVK_BLOCKS><<<tetBlocks + cBlocks, bs, 0, stream>>>(td, pos(), cd, contact_resistance, inv_h2, inv_h, inv_h2_d, tetBlocks, partials);
      break;
    default:
      k_residual_partials<R, MAT_STVK_LAME><<<tetBlocks + cBlocks, bs, 0, stream>>>(td, pos(), cd, contact_resistance, inv_h2, inv_h, inv_h2_d, tetBlocks, partials);
  }
  CU(cudaGetLastError());
  int dBlocks = 0;
  if (dc && dc->nobs) CHECK(contact_residual_partials(*dc, contact_resistance, h, partials + tetBlocks + cBlocks, &dBlocks));
  k_finish_norm<256><<<1, 256, 0, stream>>>(partials, tetBlocks + cBlocks + dBlocks, d_scalar.as<double>());
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(h_scalar.p, d_scalar.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  *out = h_scalar.as<double>()[0];
  return MLX_OK;
}

template <typename R>
int Solver<R>::norm_resv(double* out) {
  const int bs = 256;
  int grid = std::min(blocks_for(N, bs), 296);
  k_norm3_partials<R><<<grid, bs, 0, stream>>>(d_resv.as<R4<R>>(), N, d_partials.as<double>());
  CU(cudaGetLastError());
  k_finish_norm<256><<<1, 256, 0, stream>>>(d_partials.as<double>(), grid, d_scalar.as<double>() + 1);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(h_scalar.as<double>() + 1, d_scalar.as<double>() + 1, sizeof(double), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  *out = h_scalar.as<double>()[1];
  return MLX_OK;
}

template <typename R>
int Solver<R>::validate_layers(const mlx_layer_desc* ld, const mlx_solve_params* P) {
  if (!ld || !P) return set_error(MLX_ERR_ARGUMENT, "null argument");
  if (ld->num_layers < 0 || ld->num_columns < 1) return set_error(MLX_ERR_ARGUMENT, "bad layer counts");
  if (ld->num_layers > 0 && (!ld->layers_map || !ld->iterations || !ld->is_elastic_element ||
                             !ld->is_rigid_element || !ld->vertex_rigid_body || !ld->is_boundary_vertex ||
                             !ld->is_rigid_vertex || !ld->num_rigids))
    return set_error(MLX_ERR_ARGUMENT, "layer description has NULL arrays");
  if (P->run_until >= 0 && !P->compute_residuals)
    return set_error(MLX_ERR_ARGUMENT, "run_until >= 0 needs compute_residuals (the reference loop would never end)");
  if (!(P->h > 0)) return set_error(MLX_ERR_ARGUMENT, "h must be > 0");
  for (int l = 0; l < ld->num_layers; ++l) {
    if (ld->layers_map[l] < 1 || ld->layers_map[l] > ld->num_columns)
      return set_error(MLX_ERR_ARGUMENT, "layers_map entry out of range");
    if (ld->iterations[l] < 0) return set_error(MLX_ERR_ARGUMENT, "iterations must be >= 0");
  }
  return MLX_OK;
}

template <typename R>
int Solver<R>::upload_contacts(const mlx_contacts* K, ContactData& cd) {
  const int nK = (K && K->num_contacts > 0) ? K->num_contacts : 0;
  cd = ContactData{};
  cd.K = nK;
  if (nK == 0) return MLX_OK;
  if (!K->normals || !K->point_colliders || !K->vertex_ids || !K->compliance)
    return set_error(MLX_ERR_ARGUMENT, "contact arrays are NULL");
  for (int k = 0; k < nK; ++k)
    if (K->vertex_ids[k] < 1 || K->vertex_ids[k] > N) return set_error(MLX_ERR_ARGUMENT, "contact vertex id out of range");
  // the distinct compliances and their counts (the residual's K x K term)
  double cv[kMaxCompliances];
  int cn[kMaxCompliances];
  int nc = 0;
  for (int k = 0; k < nK && nc >= 0; ++k) {
    const double a = K->compliance[k];
    int g = 0;
    while (g < nc && !(cv[g] == a)) ++g;
    if (g == nc) {
      if (nc == kMaxCompliances) {
        nc = -1;
        break;
      }
      cv[nc] = a;
      cn[nc++] = 0;
    }
    ++cn[g];
  }
  // host staging: 7 nK doubles, nK ids (rounded up to whole doubles), the
  // compliance values, their counts
  const size_t o_cv = 7 * (size_t)nK + (nK + 1) / 2;
  CHECK(h_cstage.ensure(sizeof(double) * (o_cv + kMaxCompliances) + sizeof(int) * kMaxCompliances, true));
  CHECK(d_contacts.ensure(sizeof(double) * (7 * nK + kMaxCompliances) + sizeof(int) * kMaxCompliances, true));
  CHECK(d_cvid.ensure(sizeof(int) * nK, true));
  CHECK(d_clam.ensure(sizeof(double) * nK, true));
  double* hc = h_cstage.as<double>();
  host_copy(hc, K->normals, sizeof(double) * 3 * nK);
  host_copy(hc + 3 * nK, K->point_colliders, sizeof(double) * 3 * nK);
  host_copy(hc + 6 * nK, K->compliance, sizeof(double) * nK);
  int* hv = reinterpret_cast<int*>(hc + 7 * nK);
  for (int k = 0; k < nK; ++k) hv[k] = K->vertex_ids[k] - 1;
  double* hcv = hc + o_cv;
  int* hcn = reinterpret_cast<int*>(hcv + kMaxCompliances);
  for (int g = 0; g < std::max(nc, 0); ++g) {
    hcv[g] = cv[g];
    hcn[g] = cn[g];
  }
  CU(cudaMemcpyAsync(d_contacts.p, hc, sizeof(double) * 7 * nK, cudaMemcpyHostToDevice, stream));
  double* dcv = d_contacts.as<double>() + 7 * (size_t)nK;
  if (nc > 0)
    CU(cudaMemcpyAsync(dcv, hcv, sizeof(double) * kMaxCompliances + sizeof(int) * kMaxCompliances,
                       cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_cvid.p, hv, sizeof(int) * nK, cudaMemcpyHostToDevice, stream));
  CU(cudaMemsetAsync(d_clam.p, 0, sizeof(double) * nK, stream));
  cd.normal = d_contacts.as<double>();
  cd.point = cd.normal + 3 * nK;
  cd.compliance = cd.normal + 6 * nK;
  cd.vid = d_cvid.as<int>();
  cd.lambda = d_clam.as<double>();
  cd.ncomp = std::max(nc, 0);
  cd.comp_vals = dcv;
  cd.comp_counts = reinterpret_cast<const int*>(dcv + kMaxCompliances);
  return MLX_OK;
}

// One monitored iteration's residual and stop rules in one launch (no device
// contacts): every CTA writes its partial sum of the tets' residual terms;
// the last CTA to finish (ticket) sums the partials in index order exactly
// as k_finish_norm does, stores the norm and applies the monitor's rules,
// then resets the ticket for the next iteration.
template <typename R, int MAT>
__global__ void __launch_bounds__(256) k_residual_monitor(TetData<R> td, const R4<R>* __restrict__ pos, R inv_h2,
                                                          R inv_h, double inv_h2_d, double* __restrict__ partials,
                                                          unsigned* __restrict__ ticket, MonState* ms,
                                                          cudaGraphConditionalHandle loop, int iterations, int is_last,
                                                          MonParams mp, cudaGraphConditionalHandle ns, int ns_every) {
  double acc[1] = {residual_tets<R, MAT>(td, pos, inv_h2, inv_h, inv_h2_d, blockIdx.x * blockDim.x + threadIdx.x,
                                         gridDim.x * blockDim.x)};
  block_sum<1>(acc);
  __shared__ int last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = acc[0];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double sum[1] = {0.0};
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) sum[0] += __ldcg(partials + i);
  block_sum<1>(sum);
  if (threadIdx.x == 0) {
    ms->res = sqrt(sum[0]);
    *ticket = 0;
    mon_iter_end(ms, loop, iterations, is_last, mp, ns, ns_every);
  }
}

// The layer loop of layerSolve (xpbdLayer3D.m:109-226) on the device-resident
// state (pos, resv, oldp, lambda, pinned values).  With `capturing` set the
// loop issues only stream work (no host synchronisation), so it can be
// recorded into a CUDA graph; residual monitoring needs the host and is
// refused in that mode.
template <typename R>
int Solver<R>::run_layers(const mlx_layer_desc* ld, const mlx_solve_params* P, const mlx_contacts* K,
                          const ContactData& cd, RunState& st, bool capturing, LayerWork& w,
                          const DevContacts& dc) {
  // In a captured step the residual monitor runs on the device: every layer
  // is a conditional IF node and its projectGS loop a conditional WHILE node
  // (monitor.cuh).  Kernels keep plain stream order there.
  const bool devmon = capturing && P->compute_residuals;
  if (devmon && cd.K > 0)
    return set_error(MLX_ERR_UNSUPPORTED, "device residual monitoring covers device-detected contacts only");
  struct Guard {
    Solver* s;
    cudaStream_t outer;
    bool pdl;
    ~Guard() {
      for (cudaStream_t b : {s->cs_ns, s->cs_while, s->cs_if}) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (b && cudaStreamIsCapturing(b, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
          cudaGraph_t g = nullptr;
          cudaStreamEndCapture(b, &g);
        }
      }
      s->stream = outer;
      s->pdl = pdl;
    }
  } guard{this, stream, pdl};
  if (devmon) {
    // programmatic dependent launches stay on inside the conditional bodies
    // (same results; ~25 % less time per monitored iteration on config 2)
    if (!cs_if) CU(cudaStreamCreateWithFlags(&cs_if, cudaStreamNonBlocking));
    if (!cs_while) CU(cudaStreamCreateWithFlags(&cs_while, cudaStreamNonBlocking));
    if (!cs_ns) CU(cudaStreamCreateWithFlags(&cs_ns, cudaStreamNonBlocking));
  }
  MonParams mp{P->stop_at_improvement_percent, P->give_up_threshold, P->give_up_enabled,
               P->last_layer_give_up_enabled, (long long)P->hanging_stop};
  const cudaStream_t outer = stream;
  const double h = P->h;
  const R hR = (R)h;
  const int nK = cd.K;
  const size_t np = pinned.size();
  bool errorChangeDecreased = false;
  while ((int)w.cache.size() < ld->num_columns) w.cache.emplace_back(new LayerStatic());
  const long long kSafetyIterations = 100000000LL;

  for (int layer = 0; layer < ld->num_layers; ++layer) {
    double setPercentStop = layer == 0 ? P->stop_at_improvement_percent : 0;
    bool isLast = layer == ld->num_layers - 1;
    int col = ld->layers_map[layer] - 1;
    LayerStatic& ls = *w.cache[col];
    CHECK(build_static(ld, col, ls, capturing));
    const int* dint = ls.dev.as<int>();
    LayerDev L{};
    L.nb = ls.nb;
    L.body_vert_off = dint + ls.o_bvo;
    L.body_verts = dint + ls.o_bv;
    L.bnd_off = dint + ls.o_bo;
    L.bnd_verts = dint + ls.o_bnd;
    L.vert_body = dint + ls.o_vb;
    L.vert_rigid = ls.dev_rigid.as<unsigned char>();
    L.any_boundary = ls.n_bnd > 0;
    L.n_items = ls.n_items;
    L.items = dint + ls.o_items;
    // contact lists of this layer
    if (nK > 0) {
      const int32_t* rid = ls.rid.data();
      std::vector<int> rc_off(ls.nb + 1, 0), rc_ids;
      if (P->use_rigid_contacts) {
        for (int k = 0; k < nK; ++k) {
          int b = rid[K->vertex_ids[k] - 1];
          if (b > 0) ++rc_off[b];
        }
        for (int b = 1; b <= ls.nb; ++b) rc_off[b] += rc_off[b - 1];
        rc_ids.resize(rc_off[ls.nb]);
        std::vector<int> f(rc_off.begin(), rc_off.end() - 1);
        for (int k = 0; k < nK; ++k) {
          int b = rid[K->vertex_ids[k] - 1];
          if (b > 0) rc_ids[f[b - 1]++] = k;
        }
      }
      // elastic contacts grouped by vertex, groups in ascending vertex order
      // (a vertex's contacts keep their list order; groups are independent)
      std::vector<int> vcnt(N, 0), ec_off{0}, ec_vert, ec_ids;
      for (int k = 0; k < nK; ++k) {
        const int v = K->vertex_ids[k] - 1;
        if (rid[v] == 0) ++vcnt[v];
      }
      for (int v = 0; v < N; ++v)
        if (vcnt[v]) {
          ec_vert.push_back(v);
          ec_off.push_back(ec_off.back() + vcnt[v]);
          vcnt[v] = ec_off[ec_off.size() - 2];  // now the group's next free slot
        }
      const int ng = (int)ec_vert.size();
      ec_ids.resize(ec_off[ng]);
      for (int k = 0; k < nK; ++k) {
        const int v = K->vertex_ids[k] - 1;
        if (rid[v] == 0) ec_ids[vcnt[v]++] = k;
      }
      size_t o_rco = 0, o_rci = rc_off.size(), o_eco = o_rci + rc_ids.size(), o_eci = o_eco + ec_off.size(),
             o_ecv = o_eci + ec_ids.size();
      // the lists go through pinned memory that no copy in flight reads: each
      // layer of a call takes a new range (reset once the call has synchronised)
      const size_t need = o_ecv + ec_vert.size();
      if (cpack_used + need > h_cpack.bytes / sizeof(int)) {
        CU(cudaStreamSynchronize(stream));
        CHECK(h_cpack.ensure(sizeof(int) * std::max(need, 2 * (h_cpack.bytes / sizeof(int)))));
        cpack_used = 0;
      }
      int* cpack = h_cpack.as<int>() + cpack_used;
      cpack_used += need;
      std::copy(rc_off.begin(), rc_off.end(), cpack + o_rco);
      std::copy(rc_ids.begin(), rc_ids.end(), cpack + o_rci);
      std::copy(ec_off.begin(), ec_off.end(), cpack + o_eco);
      std::copy(ec_ids.begin(), ec_ids.end(), cpack + o_eci);
      std::copy(ec_vert.begin(), ec_vert.end(), cpack + o_ecv);
      CHECK(d_cgroups.ensure(sizeof(int) * need, true));
      CU(cudaMemcpyAsync(d_cgroups.p, cpack, sizeof(int) * need, cudaMemcpyHostToDevice, stream));
      const int* dc = d_cgroups.as<int>();
      L.rc_off = dc + o_rco;
      L.rc_ids = dc + o_rci;
      L.any_rigid_contact = rc_ids.size() > 0;
      L.n_ec_groups = ng;
      L.ec_off = dc + o_eco;
      L.ec_ids = dc + o_eci;
      L.ec_vert = dc + o_ecv;
    }
    const bool rigidLayer = ls.n_rigid_elements > 0;
    R4<R>* p = pos();
    R4<R>* resv = d_resv.as<R4<R>>();
    R4<R>* xprev = d_xprev.as<R4<R>>();
    double4* ri = d_ri.as<double4>();
    if (devmon) {
      // the layer runs only while stopSolve is unset
      cudaGraphConditionalHandle h_if;
      CHECK(cond_handle(&h_if));
      k_mon_layer_begin<<<1, 1, 0, stream>>>(mon(), h_if, layer, mp);
      CU(cudaGetLastError());
      ++st.launches;
      CHECK(cond_begin(h_if, cudaGraphCondTypeIf, cs_if));
    }
    if (rigidLayer && ls.nb > 0) CU(cudaMemcpyAsync(xprev, p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
    if (ls.nb > 0) {
      if (!capturing) CHECK(w.bodies.ensure(sizeof(Body) * ls.nb));
      else if (w.bodies.bytes < sizeof(Body) * ls.nb) return set_error(MLX_ERR_ARGUMENT, "body buffer not reserved");
      k_make_rigids<R><<<ls.n_items, kBodyThreads, 0, stream>>>(L, w.bodies.as<Body>(), p, resv, d_vmass.as<double>(), ri);
      CU(cudaGetLastError());
      ++st.launches;
      if (&w == &sim_work && col == ws.col && layer == 0 && (ws.record || ws.mode)) {
        CHECK(ws_after_make_rigids(w));
        st.launches += ws.mode == 1 ? 8 : 4;
      }
    }
    k_release_elastic<R><<<blocks_for(N, 256), 256, 0, stream>>>(p, resv, L.vert_rigid, N, hR);
    CU(cudaGetLastError());
    ++st.launches;
    if (rigidLayer && ls.nb > 0) {
      k_rigid_step<R><<<ls.n_items, kBodyThreads, 0, stream>>>(L, w.bodies.as<Body>(), p, xprev, resv, ri, h);
      CU(cudaGetLastError());
      ++st.launches;
    }
    double normresv = 0;
    if (devmon) {
      CHECK(norm_resv_dev(&mon()->normresv));
      st.launches += 2;
    } else if (P->compute_residuals) {
      CU(cudaStreamSynchronize(stream));
      auto t0 = std::chrono::steady_clock::now();
      CHECK(norm_resv(&normresv));
      st.sumNonMon += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    // contact multipliers restart at zero in every layer: projectGS does not
    // return them (xpbdLayer3D.m:163), so each layer sees layerSolve's zeros
    if (nK > 0) CU(cudaMemsetAsync(cd.lambda, 0, sizeof(double) * nK, stream));
    if (dc.nobs) CU(cudaMemsetAsync(dc.lambda, 0, sizeof(double) * (size_t)N * dc.nobs, stream));
    if (ls.n_bnd > 0) {
      if (!capturing) CHECK(w.lamB.ensure(sizeof(double) * ls.n_bnd));
      else if (w.lamB.bytes < sizeof(double) * ls.n_bnd) return set_error(MLX_ERR_ARGUMENT, "boundary buffer not reserved");
      CU(cudaMemsetAsync(w.lamB.p, 0, sizeof(double) * ls.n_bnd, stream));
      if (&w == &sim_work && col == ws.col && layer == 0 && ws.mode) {
        CHECK(ws_after_lamb_reset(w));
        ++st.launches;
      }
    }
    if (&w == &sim_work && isLast && mws.on) {
      CHECK(mws_start());
      st.launches += C;
    }
    // the PCG in the layer solve: a Newton-PCG correction before the last
    // layer's Gauss-Seidel and every ns_every of its iterations
    const bool nsLayer = isLast && ns_iters > 0 && mat_kind == MAT_NH && ls.nb == 0 && ls.n_rigid_elements == 0;
    if (nsLayer) CHECK(ns_correct(h, &st.launches));
    const int* dlist = dint + ls.o_list;
    const bool bodyWork = (ls.nb > 0 && (L.any_boundary || (P->use_rigid_contacts && L.any_rigid_contact))) ||
                          L.n_ec_groups > 0 || dc.nobs > 0;
    // device-detected contacts: their number is only known on the device, so
    // the extra CTAs stride over it
    const int ecBlocks = dc.nobs ? std::max(1, std::min(blocks_for(N, kBodyThreads), 296))
                                 : blocks_for(L.n_ec_groups, kBodyThreads);
    bool stopSolve = false;
    if ((persistent || (cluster_ok && ls.cl_ok)) && !P->compute_residuals && !dc.nobs) {
      // fixed iteration count: the whole projectGS loop of the layer in one launch
      const int iters = std::max(ld->iterations[layer], 0);
      if (iters > 0) {
        const bool timed = sweep_timing && tev_used + 2 <= tev.size();
        if (timed) CHECK(record_event(tev[tev_used], capturing));
        if (persistent) CHECK(launch_persistent(ls, dint, L, cd, P, iters, bodyWork, w));
        else CHECK(launch_cluster(ls, dint, L, cd, P, iters, bodyWork, w));
        if (timed) {
          double b = 0;
          for (int c = 0; c < C; ++c) b += ls.color_count[c] * (bytes_per_tet() + (ls.identity_list ? 0.0 : 4.0));
          CHECK(record_event(tev[tev_used + 1], capturing));
          tev_bytes[tev_used / 2] = b * iters;
          tev_launches[tev_used / 2] = 1;
          tev_used += 2;
        }
        ++st.launches;
        st.totalIterations += iters;
      }
      if (ls.nb > 0) {
        k_finish_layer<R><<<ls.n_items, kBodyThreads, 0, stream>>>(L, w.bodies.as<Body>(), p, resv, ri, rigidLayer ? 1 : 0);
        CU(cudaGetLastError());
        ++st.launches;
      }
      continue;
    }
    if (groups_ok && ls.gr_ok && ls.nb == 0 && !P->compute_residuals && (gr_cs == 1 || (!dc.nobs && nK == 0))) {
      // a body-free layer with a fixed iteration count: one launch, a CTA per
      // group of components
      const int iters = std::max(ld->iterations[layer], 0);
      if (iters > 0) {
        const bool timed = sweep_timing && tev_used + 2 <= tev.size();
        if (timed) CHECK(record_event(tev[tev_used], capturing));
        const HostContactGroups hcg{cd, L.ec_off, L.ec_ids, L.ec_vert, L.n_ec_groups};
        CHECK(launch_groups(ls, dint, P, iters, dc, nK > 0 ? &hcg : nullptr));
        if (timed) {
          double b = 0;
          for (int c = 0; c < C; ++c) b += ls.color_count[c] * (group_bytes_per_tet() + (ls.identity_list ? 0.0 : 4.0));
          CHECK(record_event(tev[tev_used + 1], capturing));
          tev_bytes[tev_used / 2] = b * iters + 2.0 * (double)N * sizeof(R4<R>);
          tev_launches[tev_used / 2] = 1;
          tev_used += 2;
        }
        ++st.launches;
        st.totalIterations += iters;
      }
      continue;
    }
    cudaGraphConditionalHandle h_while_cur = 0;
    if (devmon) {
      // the projectGS loop as a WHILE node whose body is one iteration
      CHECK(cond_handle(&h_while_cur));
      k_mon_loop_begin<<<1, 1, 0, stream>>>(mon(), h_while_cur, ld->iterations[layer], isLast ? 1 : 0);
      CU(cudaGetLastError());
      ++st.launches;
      CHECK(cond_begin(h_while_cur, cudaGraphCondTypeWhile, cs_while));
    }
    long long it = 1;
    while (devmon || it <= ld->iterations[layer] || (!stopSolve && st.runUntil >= 0 && isLast)) {
      // (in the device-monitored loop the correction closes the WHILE body
      // instead, below)
      if (nsLayer && ns_every > 0 && !devmon && it > 1 && (it - 1) % ns_every == 0)
        CHECK(ns_correct(h, &st.launches));
      ++it;
      if (it > kSafetyIterations) return set_error(MLX_ERR_LIMIT, "iteration safety limit reached");
      ++st.totalIterations;
      const bool timed = !devmon && sweep_timing && tev_used + 2 <= tev.size();
      if (timed) CHECK(record_event(tev[tev_used], capturing));
      long long sweep_l = 0;
      double sweep_b = 0;
      for (int c = 0; c < C; ++c) {
        if (ls.color_count[c] == 0 && !dc.colored) continue;
        CHECK(launch_color(c, ls, dlist, hR, 0, dc.colored ? &dc : nullptr, L.vert_body, h, P->contact_resistance));
        ++st.launches;
        ++sweep_l;
        sweep_b += ls.color_count[c] * (bytes_per_tet() + (ls.identity_list ? 0.0 : 4.0));
      }
      if (timed) {
        CHECK(record_event(tev[tev_used + 1], capturing));
        tev_bytes[tev_used / 2] = sweep_b;
        tev_launches[tev_used / 2] = sweep_l;
        tev_used += 2;
      }
      if (bodyWork) {
        cudaLaunchConfig_t cfg = pdl_config((ls.nb > 0 ? ls.n_items : 0) + ecBlocks, kBodyThreads);
        cudaLaunchAttribute attr = pdl_attr();
        cfg.attrs = &attr;
        cfg.numAttrs = pdl ? 1 : 0;
        CU(cudaLaunchKernelEx(&cfg, k_iterate_bodies<R>, L, w.bodies.as<Body>(), p, (const double4*)ri,
                              (const double*)d_vmass.as<double>(), w.lamB.as<double>(), cd, h,
                              P->boundary_compliance, P->contact_resistance, (int)P->use_rigid_contacts, dc,
                              (const R4<R>*)d_oldp.as<R4<R>>()));
        ++st.launches;
      }
      if (np) {
        cudaLaunchConfig_t cfg = pdl_config(blocks_for((long long)np, 256), 256);
        cudaLaunchAttribute attr = pdl_attr();
        cfg.attrs = &attr;
        cfg.numAttrs = pdl ? 1 : 0;
        CU(cudaLaunchKernelEx(&cfg, k_pin<R>, p, (const int*)d_pin_dofs.as<int>(), (const R*)d_pinx.as<R>(), (int)np));
        ++st.launches;
      }
      bool endLayer = false;
      // device-monitored last layer with corrections: the iteration's
      // monitor also sets the condition of the correction that closes the
      // WHILE body (after every ns_every iterations, when the loop goes on)
      const bool nsGate = devmon && nsLayer && ns_every > 0;
      cudaGraphConditionalHandle h_ns = 0;
      if (nsGate) CHECK(cond_handle(&h_ns));
      const int nsEvery = nsGate ? ns_every : 0;
      auto close_body = [&]() -> int {
        if (nsGate) {
          CHECK(cond_begin(h_ns, cudaGraphCondTypeIf, cs_ns));
          CHECK(ns_correct(h, &st.launches));
          CHECK(cond_end(cs_while));
        }
        return cond_end(cs_if);  // end of the WHILE body
      };
      if (devmon && !dc.nobs) {
        // residual, its norm and the stop rules in one launch
        const int tb = std::min(blocks_for(T, 256), 592);
        const R ih2 = R(1) / (hR * hR), ih = R(1) / hR;
        TetData<R> td = tets();
        double* parts = d_partials.as<double>();
        unsigned* ticket = reinterpret_cast<unsigned*>(d_scalar.as<double>() + 7);
        MonState* ms = mon();
        const int its = ld->iterations[layer], il = isLast ? 1 : 0;
        switch (mat_kind) {
          case MAT_NH:
            k_residual_monitor<R, MAT_NH><<<tb, 256, 0, stream>>>(td, pos(), ih2, ih, 1.0 / (h * h), parts, ticket, ms,
                                                                  h_while_cur, its, il, mp, h_ns,
                                                                  nsEvery);
            break;
          case MAT_STVK_BLOCKS:
            k_residual_monitor<R, MAT_STVK_BLOCKS><<<tb, 256, 0, stream>>>(td, pos(), ih2, ih, 1.0 / (h * h), parts,
                                                                           ticket, ms, h_while_cur, its, il, mp, h_ns,
                                                                  nsEvery);
            break;
          default:
            k_residual_monitor<R, MAT_STVK_LAME><<<tb, 256, 0, stream>>>(td, pos(), ih2, ih, 1.0 / (h * h), parts,
                                                                         ticket, ms, h_while_cur, its, il, mp, h_ns,
                                                                  nsEvery);
        }
        CU(cudaGetLastError());
        ++st.launches;
        CHECK(close_body());
        break;
      }
      if (devmon) {
        CHECK(residual_dev(&mon()->res, dc));
        if (dc.nobs) ++st.launches;
        k_mon_iter_end<<<1, 1, 0, stream>>>(mon(), h_while_cur, ld->iterations[layer], isLast ? 1 : 0, mp, h_ns,
                                            nsEvery);
        CU(cudaGetLastError());
        st.launches += 3;
        CHECK(close_body());
        break;
      }
      if (P->compute_residuals) {
        CU(cudaStreamSynchronize(stream));
        auto t0 = std::chrono::steady_clock::now();
        double newRes = 0;
        CHECK(residual(cd, P->contact_resistance, h, &newRes, &dc));
        st.launches += dc.nobs ? 3 : 2;
        std::vector<double>& ra = st.residualArray;
        ra.push_back(newRes);
        double lastResidual = std::fabs(ra[ra.size() - 2]);
        double newResidual = std::fabs(newRes);
        double errorChange = newResidual - lastResidual;
        if (setPercentStop > 0) {
          st.runUntil = std::max((1 - setPercentStop / 100.0) * newResidual, 1e-8);
          setPercentStop = 0;
        }
        if (errorChange < 0) errorChangeDecreased = true;
        if (P->give_up_enabled && errorChange > P->give_up_threshold && errorChangeDecreased &&
            (!isLast || P->last_layer_give_up_enabled))
          endLayer = true;
        bool stopHanging = (long long)ra.size() > P->hanging_stop && P->hanging_stop >= 0;
        if (stopHanging || (st.runUntil >= 0 && (st.runUntil >= newResidual && (isLast || normresv < st.runUntil))))
          stopSolve = true;
        st.sumNonMon += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      }
      if (endLayer || stopSolve) break;
    }
    if (ls.nb > 0) {
      k_finish_layer<R><<<ls.n_items, kBodyThreads, 0, stream>>>(L, w.bodies.as<Body>(), p, resv, ri, rigidLayer ? 1 : 0);
      CU(cudaGetLastError());
      ++st.launches;
    }
    if (devmon) CHECK(cond_end(outer));  // end of the layer's IF body
    if (stopSolve) break;
  }
  return MLX_OK;
}

// A conditional handle of the graph the solver's stream is capturing into.
template <typename R>
int Solver<R>::cond_handle(cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  CU(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &g, nullptr, nullptr));
  if (cs != cudaStreamCaptureStatusActive) return set_error(MLX_ERR_ARGUMENT, "conditional node outside a capture");
  CU(cudaGraphConditionalHandleCreate(h, g, 0, 0));
  return MLX_OK;
}

// Appends a conditional node after the captured work so far and continues
// the capture inside its body on `body` (the solver's stream becomes `body`).
template <typename R>
int Solver<R>::cond_begin(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, cudaStream_t body) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  CU(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CU(cudaGraphAddNode(&node, g, deps, nd, &np));
  CU(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
  CU(cudaStreamBeginCaptureToGraph(body, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  stream = body;
  return MLX_OK;
}

template <typename R>
int Solver<R>::cond_end(cudaStream_t parent) {
  cudaGraph_t g = nullptr;
  CU(cudaStreamEndCapture(stream, &g));
  stream = parent;
  return MLX_OK;
}

template <typename R>
int Solver<R>::residual_dev(double* out, const DevContacts& dc) {
  const int bs = 256;
  const int tetBlocks = std::min(blocks_for(T, bs), 592);
  ContactData cd{};
  const R inv_h2 = R(1) / ((R)sim.P.h * (R)sim.P.h), inv_h = R(1) / (R)sim.P.h;
  const double inv_h2_d = 1.0 / (sim.P.h * sim.P.h);
  TetData<R> td = tets();
  double* partials = d_partials.as<double>();
  switch (mat_kind) {
    case MAT_NH:
      k_residual_partials<R, MAT_NH><<<tetBlocks, bs, 0, stream>>>(td, pos(), cd, 0.0, inv_h2, inv_h, inv_h2_d, tetBlocks, partials);
      break;
    case MAT_STVK_BLOCKS:
      k_residual_partials<R, MAT_STVK_BLOCKS><<<tetBlocks, bs, 0, stream>>>(td, pos(), cd, 0.0, inv_h2, inv_h, inv_h2_d, tetBlocks, partials);
      break;
    default:
      k_residual_partials<R, MAT_STVK_LAME><<<tetBlocks, bs, 0, stream>>>(td, pos(), cd, 0.0, inv_h2, inv_h, inv_h2_d, tetBlocks, partials);
  }
  CU(cudaGetLastError());
  int dBlocks = 0;
  if (dc.nobs) CHECK(contact_residual_partials(dc, sim.P.contact_resistance, sim.P.h, partials + tetBlocks, &dBlocks));
  k_finish_norm<256><<<1, 256, 0, stream>>>(partials, tetBlocks + dBlocks, out);
  CU(cudaGetLastError());
  return MLX_OK;
}

template <typename R>
int Solver<R>::contact_residual_partials(const DevContacts& dc, double contact_resistance, double h,
                                         double* partials, int* nblocks) {
  // the number of contacts is only known on the device: a fixed grid strides over it
  const int blocks = std::max(1, std::min(blocks_for(N, 256), 64));
  k_contact_residual_partials<R><<<blocks, 256, 0, stream>>>(dc, pos(), d_oldp.as<R4<R>>(), contact_resistance,
                                                             1.0 / (h * h), partials);
  CU(cudaGetLastError());
  *nblocks = blocks;
  return MLX_OK;
}

template <typename R>
int Solver<R>::norm_resv_dev(double* out) {
  const int bs = 256;
  const int grid = std::min(blocks_for(N, bs), 296);
  k_norm3_partials<R><<<grid, bs, 0, stream>>>(d_resv.as<R4<R>>(), N, d_partials.as<double>());
  CU(cudaGetLastError());
  k_finish_norm<256><<<1, 256, 0, stream>>>(d_partials.as<double>(), grid, out);
  CU(cudaGetLastError());
  return MLX_OK;
}

template <typename R>
int Solver<R>::reset_gsync() {
  CU(cudaMemsetAsync(d_gsync.p, 0, sizeof(unsigned int) * 4, stream));
  return MLX_OK;
}

// Copies the barrier error flag to the host (stream-ordered); check_gsync
// reads it after the stream has been synchronised.
template <typename R>
int Solver<R>::check_gsync() {
  if (h_gsync.as<int>()[2] != 0)
    return set_error(MLX_ERR_LIMIT, "a grid barrier of the persistent layer kernel waited more than 1 s");
  return MLX_OK;
}

template <typename R>
int Solver<R>::launch_persistent(const LayerStatic& ls, const int* dint, const LayerDev& L, const ContactData& cd,
                                 const mlx_solve_params* P, int iterations, bool body_work, LayerWork& w) {
  PersistArgs pa;
  pa.list = ls.identity_list ? nullptr : dint + ls.o_list;
  pa.cstart = dint + ls.o_cstart;
  pa.ccount = dint + ls.o_ccount;
  pa.C = C;
  pa.iterations = iterations;
  pa.body_work = body_work ? 1 : 0;
  pa.pin_dofs = d_pin_dofs.as<int>();
  pa.npin = (int)pinned.size();
  int maxc = 0;
  for (int c = 0; c < C; ++c) maxc = std::max(maxc, ls.color_count[c]);
  pa.one_per_thread = maxc <= persist_ctas * 128 ? 1 : 0;
  GridSync gs;
  gs.count = d_gsync.as<unsigned int>();
  gs.error = reinterpret_cast<int*>(d_gsync.as<unsigned int>() + 2);
  const R hR = (R)P->h;
  const R inv_h2 = R(1) / (hR * hR), inv_h = R(1) / hR;
  TetData<R> td = tets();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(persist_ctas);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // the arrival counter restarts at zero for every launch (barrier k of a
  // launch waits for k * grid arrivals); the error flag is kept for the step
  CU(cudaMemsetAsync(d_gsync.p, 0, sizeof(unsigned int), stream));
  Body* bodies = w.bodies.as<Body>();
  double* lamB = w.lamB.as<double>();
  const double4* ri = d_ri.as<double4>();
  const R4<R>* oldp = d_oldp.as<R4<R>>();
  const double* vm = d_vmass.as<double>();
  const R* pv = d_pinx.as<R>();
  const double h = P->h;
  cudaError_t e;
  switch (mat_kind) {
    case MAT_NH:
      e = cudaLaunchKernelEx(&cfg, k_layer_persistent<R, MAT_NH, false>, td, pa, pos(), oldp, inv_h2, inv_h, L,
                             bodies, ri, vm, lamB, cd, h, P->boundary_compliance, P->contact_resistance,
                             P->use_rigid_contacts, pv, gs);
      break;
    case MAT_STVK_BLOCKS:
      e = damp ? cudaLaunchKernelEx(&cfg, k_layer_persistent<R, MAT_STVK_BLOCKS, true>, td, pa, pos(), oldp, inv_h2,
                                    inv_h, L, bodies, ri, vm, lamB, cd, h, P->boundary_compliance,
                                    P->contact_resistance, P->use_rigid_contacts, pv, gs)
               : cudaLaunchKernelEx(&cfg, k_layer_persistent<R, MAT_STVK_BLOCKS, false>, td, pa, pos(), oldp,
                                    inv_h2, inv_h, L, bodies, ri, vm, lamB, cd, h, P->boundary_compliance,
                                    P->contact_resistance, P->use_rigid_contacts, pv, gs);
      break;
    default:
      e = damp ? cudaLaunchKernelEx(&cfg, k_layer_persistent<R, MAT_STVK_LAME, true>, td, pa, pos(), oldp, inv_h2,
                                    inv_h, L, bodies, ri, vm, lamB, cd, h, P->boundary_compliance,
                                    P->contact_resistance, P->use_rigid_contacts, pv, gs)
               : cudaLaunchKernelEx(&cfg, k_layer_persistent<R, MAT_STVK_LAME, false>, td, pa, pos(), oldp,
                                    inv_h2, inv_h, L, bodies, ri, vm, lamB, cd, h, P->boundary_compliance,
                                    P->contact_resistance, P->use_rigid_contacts, pv, gs);
  }
  if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("persistent layer launch: ") + cudaGetErrorString(e));
  return MLX_OK;
}

// Vertex slots of the cluster kernel for one layer.  Every CTA keeps a slot
// for each vertex its tets touch; a tet writes its four corners into its own
// CTA's slots and reads each corner from the slot of that vertex's previous
// writer in colour order (the schedule is static, so that slot is known
// here).  Between two writers of a vertex no other tet touches it, so the
// slot still holds the value when the next writer reads it, and no tet ever
// stores into another CTA's shared memory.  A vertex's home slot is the one
// of its last writer in a sweep (the owning part's slot if no elastic tet
// touches it): the body, contact and pinning phases work there, the first
// writer of the next sweep reads from there, and the launch fills and
// drains it.
template <typename R>
int Solver<R>::build_cluster_slots(LayerStatic& ls, const std::vector<int>& list) {
  const int P = cl_size;
  const int nE = ls.identity_list ? T : (int)list.size();
  auto sid = [&](int i) { return ls.identity_list ? i : list[i]; };
  std::vector<int> slot((size_t)P * N, -1), cnt(P, 0), last(N, -1);
  for (int i = 0; i < nE; ++i) {
    const int s = sid(i), r = tpart_sorted[s];
    const int4 q = vid_sorted[s];
    for (int v : {q.x, q.y, q.z, q.w}) {
      int& sl = slot[(size_t)r * N + v];
      if (sl < 0) sl = cnt[r]++;
      last[v] = r;
    }
  }
  std::vector<int> home(N), vhome(N);
  for (int v = 0; v < N; ++v) {
    const int r = last[v] >= 0 ? last[v] : vowner[v];
    int& sl = slot[(size_t)r * N + v];
    if (sl < 0) sl = cnt[r]++;
    home[v] = r;
    vhome[v] = (r << 24) | sl;
  }
  int maxs = 0;
  for (int r = 0; r < P; ++r) maxs = std::max(maxs, cnt[r]);
  if (maxs >= 65536) {
    ls.cl_ok = false;
    return MLX_OK;
  }
  std::vector<int4> tsrc(nE);
  std::vector<int2> tdst(nE);
  std::vector<int> prev(home);
  for (int i = 0; i < nE; ++i) {
    const int s = sid(i), r = tpart_sorted[s];
    const int4 q = vid_sorted[s];
    int src[4], dst[4];
    const int vv[4] = {q.x, q.y, q.z, q.w};
    for (int k = 0; k < 4; ++k) {
      const int v = vv[k];
      src[k] = (prev[v] << 24) | slot[(size_t)prev[v] * N + v];
      dst[k] = slot[(size_t)r * N + v];
      prev[v] = r;
    }
    tsrc[i] = make_int4(src[0], src[1], src[2], src[3]);
    tdst[i] = make_int2(dst[0] | (dst[1] << 16), dst[2] | (dst[3] << 16));
  }
  std::vector<int> hoff(P + 1, 0), hv(N), hs(N);
  for (int v = 0; v < N; ++v) ++hoff[home[v] + 1];
  for (int r = 0; r < P; ++r) hoff[r + 1] += hoff[r];
  {
    std::vector<int> fill(hoff.begin(), hoff.end() - 1);
    for (int v = 0; v < N; ++v) {
      const int q = fill[home[v]]++;
      hv[q] = v;
      hs[q] = vhome[v] & 0xffffff;
    }
  }
  // shared memory: slots, then the multipliers when they fit
  const long long rec = (long long)maxs * (long long)sizeof(R4<R>);
  const int nl = mat_kind == MAT_NH ? 2 : 6;
  int lam = cl_lam_slots;
  long long smem = rec + (long long)lam * nl * (long long)sizeof(R);
  if (smem > cl_budget) {
    lam = 0;
    smem = rec;
  }
  if (smem > cl_budget) {
    ls.cl_ok = false;
    return MLX_OK;
  }
  size_t ints = 0;
  ls.o_tsrc = ints; ints += 4 * (size_t)nE;
  ls.o_tdst = ints; ints += 2 * (size_t)nE;
  ls.o_vhome = ints; ints += N;
  ls.o_hv = ints; ints += N;
  ls.o_hs = ints; ints += N;
  ls.o_hoff = ints; ints += P + 1;
  std::vector<int> pack(ints);
  std::memcpy(pack.data() + ls.o_tsrc, tsrc.data(), sizeof(int4) * nE);
  std::memcpy(pack.data() + ls.o_tdst, tdst.data(), sizeof(int2) * nE);
  std::memcpy(pack.data() + ls.o_vhome, vhome.data(), sizeof(int) * N);
  std::memcpy(pack.data() + ls.o_hv, hv.data(), sizeof(int) * N);
  std::memcpy(pack.data() + ls.o_hs, hs.data(), sizeof(int) * N);
  std::memcpy(pack.data() + ls.o_hoff, hoff.data(), sizeof(int) * (P + 1));
  CHECK(ls.cl_dev.ensure(sizeof(int) * ints));
  CU(cudaMemcpyAsync(ls.cl_dev.p, pack.data(), sizeof(int) * ints, cudaMemcpyHostToDevice, stream));
  CU(cudaStreamSynchronize(stream));
  ls.cl_slots = maxs;
  ls.cl_lam = lam;
  ls.cl_smem = (size_t)smem;
  ls.cl_ok = true;
  return MLX_OK;
}

template <typename R>
int Solver<R>::launch_cluster(const LayerStatic& ls, const int* dint, const LayerDev& L, const ContactData& cd,
                              const mlx_solve_params* P, int iterations, bool body_work, LayerWork& w) {
  ClusterArgs ca;
  ca.list = ls.identity_list ? nullptr : dint + ls.o_list;
  ca.off = dint + ls.o_cloff;
  ca.lbase = dint + ls.o_cllb;
  ca.colours = dint + ls.o_clcol;
  ca.rec_slots = ls.cl_slots;
  ca.lam_slots = ls.cl_lam;
  ca.nC = ls.cl_nC;
  const int* cl = ls.cl_dev.as<int>();
  ca.tsrc = reinterpret_cast<const int4*>(cl + ls.o_tsrc);
  ca.tdst = reinterpret_cast<const int2*>(cl + ls.o_tdst);
  ca.vhome = cl + ls.o_vhome;
  ca.home_v = cl + ls.o_hv;
  ca.home_s = cl + ls.o_hs;
  ca.home_off = cl + ls.o_hoff;
  ca.iterations = iterations;
  ca.body_work = body_work ? 1 : 0;
  ca.pin_dofs = d_pin_dofs.as<int>();
  ca.npin = (int)pinned.size();
  ca.one_per_thread = ls.cl_max_range <= cl_threads ? 1 : 0;
  const R hR = (R)P->h;
  const R inv_h2 = R(1) / (hR * hR), inv_h = R(1) / hR;
  TetData<R> td = tets();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl_size);
  cfg.blockDim = dim3(cl_threads);
  cfg.dynamicSmemBytes = ls.cl_smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  Body* bodies = w.bodies.as<Body>();
  double* lamB = w.lamB.as<double>();
  const double4* ri = d_ri.as<double4>();
  const R4<R>* oldp = d_oldp.as<R4<R>>();
  const double* vm = d_vmass.as<double>();
  const R* pv = d_pinx.as<R>();
  const double h = P->h;
  const double bc = P->boundary_compliance, cr = P->contact_resistance;
  const int urc = P->use_rigid_contacts;
  cudaError_t e;
  switch (mat_kind) {
    case MAT_NH:
      e = cudaLaunchKernelEx(&cfg, k_layer_cluster<R, MAT_NH, false>, td, ca, pos(), oldp, inv_h2, inv_h, L, bodies,
                             ri, vm, lamB, cd, h, bc, cr, urc, pv);
      break;
    case MAT_STVK_BLOCKS:
      e = damp ? cudaLaunchKernelEx(&cfg, k_layer_cluster<R, MAT_STVK_BLOCKS, true>, td, ca, pos(), oldp, inv_h2,
                                    inv_h, L, bodies, ri, vm, lamB, cd, h, bc, cr, urc, pv)
               : cudaLaunchKernelEx(&cfg, k_layer_cluster<R, MAT_STVK_BLOCKS, false>, td, ca, pos(), oldp, inv_h2,
                                    inv_h, L, bodies, ri, vm, lamB, cd, h, bc, cr, urc, pv);
      break;
    default:
      e = damp ? cudaLaunchKernelEx(&cfg, k_layer_cluster<R, MAT_STVK_LAME, true>, td, ca, pos(), oldp, inv_h2,
                                    inv_h, L, bodies, ri, vm, lamB, cd, h, bc, cr, urc, pv)
               : cudaLaunchKernelEx(&cfg, k_layer_cluster<R, MAT_STVK_LAME, false>, td, ca, pos(), oldp, inv_h2,
                                    inv_h, L, bodies, ri, vm, lamB, cd, h, bc, cr, urc, pv);
  }
  if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("cluster layer launch: ") + cudaGetErrorString(e));
  return MLX_OK;
}

template <typename R>
int Solver<R>::layer_solve(const mlx_layer_desc* ld, const mlx_solve_params* P, const mlx_contacts* K,
                           const mlx_solve_inputs* in, mlx_solve_outputs* out) {
  if (!ld || !P || !in || !out) return set_error(MLX_ERR_ARGUMENT, "null argument");
  if (!in->xi || !in->oldp || !in->residualv || !out->xi)
    return set_error(MLX_ERR_ARGUMENT, "xi, oldp, residualv and out->xi are required");
  if (!pinned.empty() && !in->pinnedx) return set_error(MLX_ERR_ARGUMENT, "pinnedx is NULL");
  CHECK(validate_layers(ld, P));
  if (in->residual_in_len < 1 && P->compute_residuals)
    return set_error(MLX_ERR_ARGUMENT, "residual_in must hold at least the initial entry");
  if (P->contact_coloring && K && K->num_contacts > 0)
    return set_error(MLX_ERR_UNSUPPORTED, "contact_coloring needs device-detected contacts (mlx_sim_set_obstacles)");

  DeviceGuard g(device);
  const size_t n3 = 3 * (size_t)N, n6 = 6 * (size_t)T, np = pinned.size();
  // ---- upload per-call vectors (one pinned staging copy) ----
  // Staged: xi, residualv, oldp when damping reads it, lambdai unless NULL
  // (all zeros, what integrate passes), the pinned values.
  const size_t o_old = 2 * n3, o_lam = o_old + (damp ? n3 : 0), o_pin = o_lam + (in->lambdai ? n6 : 0);
  const size_t nst = std::max<size_t>(o_pin + np, n3 + (out->lambdai ? n6 : 0));
  CHECK(h_stage.ensure(sizeof(double) * nst));
  CHECK(d_stage.ensure(sizeof(double) * nst));
  double* hs = h_stage.as<double>();
  double* ds = d_stage.as<double>();
  // vectors of a MB or more go up one by one, each copy overlapping the
  // staging of the next
  const bool piecewise = sizeof(double) * n3 >= (size_t(1) << 20);
  size_t sent = 0;
  auto stage = [&](size_t off, const double* src, size_t n) -> int {
    host_copy(hs + off, src, sizeof(double) * n);
    if (piecewise) {
      CU(cudaMemcpyAsync(ds + sent, hs + sent, sizeof(double) * (off + n - sent), cudaMemcpyHostToDevice, stream));
      sent = off + n;
    }
    return MLX_OK;
  };
  CHECK(stage(0, in->xi, n3));
  CHECK(stage(n3, in->residualv, n3));
  if (damp) CHECK(stage(o_old, in->oldp, n3));
  if (in->lambdai) CHECK(stage(o_lam, in->lambdai, n6));
  if (np) CHECK(stage(o_pin, in->pinnedx, np));
  if (o_pin + np > sent)
    CU(cudaMemcpyAsync(ds + sent, hs + sent, sizeof(double) * (o_pin + np - sent), cudaMemcpyHostToDevice, stream));
  const int bs = 256;
  k_load_pos<R><<<blocks_for(N, bs), bs, 0, stream>>>(ds, d_mass3.as<double>(), pos(), N);
  k_load_vec<R><<<blocks_for(N, bs), bs, 0, stream>>>(ds + n3, d_resv.as<R4<R>>(), N);
  if (damp) k_load_vec<R><<<blocks_for(N, bs), bs, 0, stream>>>(ds + o_old, d_oldp.as<R4<R>>(), N);
  if (in->lambdai)
    k_load_lambda<R><<<blocks_for(T, bs), bs, 0, stream>>>(ds + o_lam, d_s2e.as<int>(), d_lambda.as<R>(), T);
  else
    CU(cudaMemsetAsync(d_lambda.p, 0, sizeof(R) * n6, stream));
  if (np) k_cast<R><<<blocks_for((long long)np, bs), bs, 0, stream>>>(ds + o_pin, d_pinx.as<R>(), (int)np);
  CU(cudaGetLastError());
  ContactData cd;
  CHECK(upload_contacts(K, cd));

  RunState st;
  st.residualArray.assign(in->residual_in, in->residual_in + std::max(in->residual_in_len, 0));
  st.runUntil = P->run_until;
  st.sumNonMon = in->sum_non_monitored_time;
  CHECK(reset_gsync());
  // A call of the same shape as the previous one replays it as a graph; with
  // residual monitoring the stop rules then run on the device (monitor.cuh:
  // the same rules and residual bits as the host loop), the residual array
  // going in and out through the device monitor's state.  The time spent on
  // residuals is not measured there (sum_non_monitored_time passes through).
  const bool monDev = P->compute_residuals && in->residual_in_len < kMonCapacity;
  const bool graphable = host_graph_on && (!P->compute_residuals || monDev) && cd.K == 0 && !sweep_timing;
  std::vector<int> lkey;
  std::vector<unsigned char> pkey;
  if (graphable) {
    lkey = {ld->num_layers, ld->num_columns};
    for (int l = 0; l < ld->num_layers; ++l) {
      lkey.push_back(ld->layers_map[l]);
      lkey.push_back(ld->iterations[l]);
    }
    pkey.assign(reinterpret_cast<const unsigned char*>(P), reinterpret_cast<const unsigned char*>(P) + sizeof(*P));
  }
  bool replayed = false;
  if (graphable && lkey == hg.lkey && pkey == hg.pkey && statics_hit(ld, work)) {
    replayed = true;
    // the monitor's state lives at a fixed address the graph records
    if (P->compute_residuals) CHECK(d_mon_ls.ensure(sizeof(MonState)));
    // the same shape as the previous call, whose uncaptured run built every
    // layer static: record the loop once, then replay it
    if (!hg.exec) {
      cudaGraph_t graph = nullptr;
      CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      RunState cs = st;
      mon_active = &d_mon_ls;
      const int rc = run_layers(ld, P, K, cd, cs, true, work);
      mon_active = &d_mon;
      const cudaError_t e = cudaStreamEndCapture(stream, &graph);
      if (rc != MLX_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
      const cudaError_t ei = cudaGraphInstantiate(&hg.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        hg.exec = nullptr;
        return set_error(MLX_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
      }
      hg.launches = cs.launches - st.launches;
      hg.iterations = cs.totalIterations - st.totalIterations;
    }
    if (P->compute_residuals) {
      // the monitor's state for this call: the caller's residual array and
      // run-until, the rest cleared as at the start of the host loop
      CHECK(h_mon.ensure(sizeof(MonState)));
      MonState* hm = h_mon.as<MonState>();
      const size_t head = offsetof(MonState, ra);
      std::memset(static_cast<void*>(hm), 0, head);
      hm->run_until = P->run_until;
      hm->ra_len = in->residual_in_len;
      std::memcpy(hm->ra, in->residual_in, sizeof(double) * in->residual_in_len);
      CU(cudaMemcpyAsync(d_mon_ls.p, hm, head + sizeof(double) * in->residual_in_len, cudaMemcpyHostToDevice,
                         stream));
    }
    CU(cudaGraphLaunch(hg.exec, stream));
    st.launches += hg.launches;
    if (P->compute_residuals)
      CU(cudaMemcpyAsync(h_mon.p, d_mon_ls.p, sizeof(MonState), cudaMemcpyDeviceToHost, stream));
    else
      st.totalIterations += hg.iterations;
  } else {
    drop_host_graph();
    CHECK(run_layers(ld, P, K, cd, st, false, work));
    hg.lkey = lkey;
    hg.pkey = pkey;
  }
  CU(cudaMemcpyAsync(h_gsync.p, d_gsync.p, sizeof(unsigned int) * 4, cudaMemcpyDeviceToHost, stream));
  // ---- download ----
  k_store_pos<R><<<blocks_for(N, bs), bs, 0, stream>>>(pos(), ds, N);
  if (out->lambdai) k_store_lambda<R><<<blocks_for(T, bs), bs, 0, stream>>>(d_lambda.as<R>(), d_s2e.as<int>(), ds + n3, T);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(hs, ds, sizeof(double) * (out->lambdai ? n3 + n6 : n3), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  cpack_used = 0;  // no copy of the contact lists is in flight now
  CHECK(check_gsync());
  if (P->compute_residuals && replayed) {
    // replayed with the stop rules on the device
    const MonState* hm = h_mon.as<MonState>();
    if (hm->error == 1) return set_error(MLX_ERR_LIMIT, "a layer reached the device monitor's iteration cap");
    if (hm->error == 2) return set_error(MLX_ERR_LIMIT, "the residual array reached the device monitor's capacity");
    st.residualArray.assign(hm->ra, hm->ra + hm->ra_len);
    st.runUntil = hm->run_until;
    st.totalIterations = hm->total_iterations;
  }
  host_copy(out->xi, hs, sizeof(double) * n3);
  if (out->lambdai) host_copy(out->lambdai, hs + n3, sizeof(double) * n6);
  int n = (int)st.residualArray.size();
  if (out->residual) {
    if (n > out->residual_capacity) return set_error(MLX_ERR_ARGUMENT, "residual capacity too small");
    std::memcpy(out->residual, st.residualArray.data(), sizeof(double) * n);
  }
  out->residual_len = n;
  out->run_until = st.runUntil;
  out->sum_non_monitored_time = st.sumNonMon;
  out->total_iterations = st.totalIterations;
  last_launches = st.launches;
  return MLX_OK;
}

// ---------------------------------------------------------------------------
// Device-resident stepping: xpbdLayer3D.integrate (xpbdLayer3D.m:621-745) with
// a fixed layer description, no host round trip between steps.

// Step start (xpbdLayer3D.m:638-666): f = m g on z, oldp = p, residual
// velocity = v + h f/m on unpinned DOFs, times (1 - airDrag).
template <typename R>
__global__ void k_sim_begin(const R4<R>* __restrict__ pos, const R4<R>* __restrict__ vel,
                            R4<R>* __restrict__ oldp, R4<R>* __restrict__ resv,
                            const double* __restrict__ mass3, const unsigned char* __restrict__ pin_mask,
                            int N, double h, double gravity, double air) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  R4<R> p = pos[v], u = vel[v];
  oldp[v] = make_r4<R>(p.x, p.y, p.z, 0);
  unsigned char pm = pin_mask[v];
  double r[3] = {(double)u.x, (double)u.y, (double)u.z};
  double fz = 0.0 + mass3[3 * v + 2] * gravity;
  if (!(pm & 4)) r[2] = r[2] + (h * fz) / mass3[3 * v + 2];
  if (!(pm & 1)) r[0] = r[0] + (h * 0.0) / mass3[3 * v];
  if (!(pm & 2)) r[1] = r[1] + (h * 0.0) / mass3[3 * v + 1];
  double k = 1.0 - air;
  resv[v] = make_r4<R>((R)(k * r[0]), (R)(k * r[1]), (R)(k * r[2]), 0);
}

// Step end (xpbdLayer3D.m:737-738): v = (xi - oldp)/h, p = xi.
template <typename R>
__global__ void k_sim_end(const R4<R>* __restrict__ pos, const R4<R>* __restrict__ oldp,
                          R4<R>* __restrict__ vel, int N, double h) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  R4<R> p = pos[v], o = oldp[v];
  vel[v] = make_r4<R>((R)(((double)p.x - o.x) / h), (R)(((double)p.y - o.y) / h), (R)(((double)p.z - o.z) / h), 0);
}

template <typename R>
__global__ void k_add_velocity(R4<R>* __restrict__ vel, const int* __restrict__ dofs,
                               const double* __restrict__ dv, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int d = dofs[i];
  R* u = reinterpret_cast<R*>(&vel[d / 3]);
  u[d % 3] = (R)((double)u[d % 3] + dv[i]);
}

template <typename R>
int Solver<R>::sim_setup(const mlx_layer_desc* ld, const mlx_solve_params* P, const double* p0, const double* v0) {
  CHECK(validate_layers(ld, P));
  if (!p0) return set_error(MLX_ERR_ARGUMENT, "initial positions are required");
  DeviceGuard g(device);
  if (P->compute_residuals) {
    CHECK(d_mon.ensure(sizeof(MonState)));
    CU(cudaMemsetAsync(d_mon.p, 0, sizeof(MonState), stream));
    CU(cudaMemcpyAsync(&mon()->run_until, &P->run_until, sizeof(double), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
  }
  sim_last.valid = false;
  // copy the fixed layer description (the caller's arrays may go away)
  const size_t TL = (size_t)T * ld->num_columns, NL = (size_t)N * ld->num_columns;
  sim.layers_map.assign(ld->layers_map, ld->layers_map + ld->num_layers);
  sim.iterations.assign(ld->iterations, ld->iterations + ld->num_layers);
  sim.isE.assign(ld->is_elastic_element, ld->is_elastic_element + TL);
  sim.isR.assign(ld->is_rigid_element, ld->is_rigid_element + TL);
  sim.sets.assign(ld->rigid_body_sets, ld->rigid_body_sets + TL);
  sim.rid.assign(ld->vertex_rigid_body, ld->vertex_rigid_body + NL);
  sim.isBV.assign(ld->is_boundary_vertex, ld->is_boundary_vertex + NL);
  sim.isRV.assign(ld->is_rigid_vertex, ld->is_rigid_vertex + NL);
  sim.nr.assign(ld->num_rigids, ld->num_rigids + ld->num_columns);
  sim.ld = *ld;
  sim.ld.layers_map = sim.layers_map.data();
  sim.ld.iterations = sim.iterations.data();
  sim.ld.is_elastic_element = sim.isE.data();
  sim.ld.is_rigid_element = sim.isR.data();
  sim.ld.rigid_body_sets = sim.sets.data();
  sim.ld.vertex_rigid_body = sim.rid.data();
  sim.ld.is_boundary_vertex = sim.isBV.data();
  sim.ld.is_rigid_vertex = sim.isRV.data();
  sim.ld.num_rigids = sim.nr.data();
  sim.P = *P;
  // build every column once and reserve the body buffers for capture
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  sim_work.cache.clear();
  while ((int)sim_work.cache.size() < ld->num_columns) sim_work.cache.emplace_back(new LayerStatic());
  int maxb = 1, maxbnd = 1;
  for (int c = 0; c < ld->num_columns; ++c) {
    CHECK(build_static(&sim.ld, c, *sim_work.cache[c], false));
    maxb = std::max(maxb, sim_work.cache[c]->nb);
    maxbnd = std::max(maxbnd, sim_work.cache[c]->n_bnd);
  }
  CHECK(sim_work.bodies.ensure(sizeof(Body) * maxb));
  CHECK(sim_work.lamB.ensure(sizeof(double) * maxbnd));
  CHECK(d_vel.ensure(sizeof(R4<R>) * N));
  CHECK(d_pin_mask.ensure(N));
  std::vector<unsigned char> pm(N, 0);
  for (int d : pinned) pm[d / 3] |= (unsigned char)(1u << (d % 3));
  // state: positions, velocities, pinned values = positions of frame 1
  const size_t n3 = 3 * (size_t)N, np = pinned.size();
  CHECK(h_stage.ensure(sizeof(double) * (2 * n3 + np)));
  CHECK(d_stage.ensure(sizeof(double) * (2 * n3 + np)));
  double* hs = h_stage.as<double>();
  std::memcpy(hs, p0, sizeof(double) * n3);
  sim_p0.assign(p0, p0 + n3);
  ws.reset();
  mws.on = 0;
  if (v0) std::memcpy(hs + n3, v0, sizeof(double) * n3);
  else std::memset(hs + n3, 0, sizeof(double) * n3);
  for (size_t i = 0; i < np; ++i) hs[2 * n3 + i] = p0[pinned[i]];
  CU(cudaMemcpyAsync(d_stage.p, hs, sizeof(double) * (2 * n3 + np), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_pin_mask.p, pm.data(), N, cudaMemcpyHostToDevice, stream));
  double* ds = d_stage.as<double>();
  k_load_pos<R><<<blocks_for(N, 256), 256, 0, stream>>>(ds, d_mass3.as<double>(), pos(), N);
  k_load_vec<R><<<blocks_for(N, 256), 256, 0, stream>>>(ds + n3, d_vel.as<R4<R>>(), N);
  if (np) k_cast<R><<<blocks_for((long long)np, 256), 256, 0, stream>>>(ds + 2 * n3, d_pinx.as<R>(), (int)np);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(stream));
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  sim.ready = true;
  return MLX_OK;
}

// Per-colour tile autotuner.  For every layer column of the resident
// stepper and every colour with elastic tets, times `reps` back-to-back
// launches of the colour kernel at each candidate block size on the current
// state and keeps the fastest; positions and multipliers are restored
// afterwards, so the simulation is unchanged.  The tuned tiles are kept only
// if a captured step with them is faster than with the default tiles.  The
// step graph is recaptured at the next step.  before_ms / after_ms
// (optional) receive one captured step's device time with the default tiles
// and with the tiles kept.
template <typename R>
int Solver<R>::sim_autotune(int reps, double* before_ms, double* after_ms) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "mlx_sim_init first");
  if (reps < 1) return set_error(MLX_ERR_ARGUMENT, "reps must be >= 1");
  DeviceGuard g(device);
  auto step_ms = [&](double* out) -> int {
    if (!out) return MLX_OK;
    DevBuf sp, sl, sv;
    CHECK(sp.ensure(sizeof(R4<R>) * N));
    CHECK(sv.ensure(sizeof(R4<R>) * N));
    CHECK(sl.ensure(sizeof(R) * 6 * (size_t)T));
    CU(cudaMemcpyAsync(sp.p, d_pos.p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
    CU(cudaMemcpyAsync(sv.p, d_vel.p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
    CU(cudaMemcpyAsync(sl.p, d_lambda.p, sizeof(R) * 6 * (size_t)T, cudaMemcpyDeviceToDevice, stream));
    if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
    double ms = 0;
    CHECK(sim_step(1, 1, nullptr));   // capture
    CHECK(sim_step(3, 1, &ms));
    *out = ms / 3;
    CU(cudaMemcpyAsync(d_pos.p, sp.p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
    CU(cudaMemcpyAsync(d_vel.p, sv.p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
    CU(cudaMemcpyAsync(d_lambda.p, sl.p, sizeof(R) * 6 * (size_t)T, cudaMemcpyDeviceToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return MLX_OK;
  };
  tiles.clear();
  for (auto& c : sim_work.cache) c->tile.clear();
  CHECK(step_ms(before_ms));
  DevBuf save_p, save_l;
  CHECK(save_p.ensure(sizeof(R4<R>) * N));
  CHECK(save_l.ensure(sizeof(R) * 6 * (size_t)T));
  CU(cudaMemcpyAsync(save_p.p, d_pos.p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
  CU(cudaMemcpyAsync(save_l.p, d_lambda.p, sizeof(R) * 6 * (size_t)T, cudaMemcpyDeviceToDevice, stream));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  const int cand[] = {32, 64, 128, 256};
  static_assert(256 <= kMaxColorTile, "autotuner candidates exceed the colour kernel's launch bound");
  const bool saved_pdl = pdl;
  pdl = false;  // isolated launches
  int rc = MLX_OK;
  tiles.assign(sim.ld.num_columns, std::vector<int>());
  const R hR = (R)sim.P.h;
  for (int col = 0; col < sim.ld.num_columns && rc == MLX_OK; ++col) {
    LayerStatic& ls = *sim_work.cache[col];
    const int* dlist = ls.dev.as<int>() + ls.o_list;
    std::vector<int> best(C, 0);
    for (int c = 0; c < C && rc == MLX_OK; ++c) {
      if (ls.color_count[c] == 0) continue;
      float best_ms = 1e30f;
      for (int bs : cand) {
        rc = launch_color(c, ls, dlist, hR, bs);  // warm-up
        if (rc != MLX_OK) break;
        cudaEventRecord(e0, stream);
        for (int r = 0; r < reps && rc == MLX_OK; ++r) rc = launch_color(c, ls, dlist, hR, bs);
        cudaEventRecord(e1, stream);
        if (rc != MLX_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = set_error(MLX_ERR_CUDA, "autotune timing failed"); break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best[c] = bs; }
      }
    }
    tiles[col] = best;
    ls.tile = best;
  }
  pdl = saved_pdl;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaMemcpyAsync(d_pos.p, save_p.p, sizeof(R4<R>) * N, cudaMemcpyDeviceToDevice, stream));
  CU(cudaMemcpyAsync(d_lambda.p, save_l.p, sizeof(R) * 6 * (size_t)T, cudaMemcpyDeviceToDevice, stream));
  CU(cudaStreamSynchronize(stream));
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  if (rc != MLX_OK) return rc;
  // keep the tiles only if the captured step (with programmatic dependent
  // launches, unlike the isolated timings above) got faster
  double before = 0, after = 0;
  CHECK(step_ms(&before));  // tuned
  const std::vector<std::vector<int>> tuned = tiles;
  tiles.clear();
  for (auto& c : sim_work.cache) c->tile.clear();
  CHECK(step_ms(&after));   // default
  if (before < after) {
    tiles = tuned;
    for (int col = 0; col < sim.ld.num_columns; ++col) sim_work.cache[col]->tile = tiles[col];
  }
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  if (after_ms) *after_ms = std::min(before, after);
  for (auto& c : work.cache) c->valid = false;  // the host-buffer path picks the tiles up on its next build
  return MLX_OK;
}

// Host preparation of the finders (their constructors): the plane's unit
// normal and offset, the box's normalised directions and half extents.
static int prepare_obstacles(const mlx_obstacle* in, int n, std::vector<Obstacle>& out) {
  if (n < 0 || n > MLX_MAX_OBSTACLES) return set_error(MLX_ERR_ARGUMENT, "num_obstacles out of [0, 32]");
  if (n > 0 && !in) return set_error(MLX_ERR_ARGUMENT, "obstacles is NULL");
  out.clear();
  for (int i = 0; i < n; ++i) {
    const mlx_obstacle& a = in[i];
    Obstacle o{};
    o.type = a.type;
    o.compliance = a.compliance;
    for (int d = 0; d < 3; ++d) o.c[d] = a.center[d];
    if (a.type == MLX_OBSTACLE_PLANE) {
      const double nn = std::sqrt(a.normal[0] * a.normal[0] + a.normal[1] * a.normal[1] + a.normal[2] * a.normal[2]);
      if (!(nn > 0)) return set_error(MLX_ERR_ARGUMENT, "plane normal is zero");
      for (int d = 0; d < 3; ++d) o.n[d] = a.normal[d] / nn;
      o.D = a.normal[0] * a.center[0] + a.normal[1] * a.center[1] + a.normal[2] * a.center[2];
    } else if (a.type == MLX_OBSTACLE_SPHERE) {
      if (!(a.radius >= 0)) return set_error(MLX_ERR_ARGUMENT, "sphere radius < 0");
      o.radius = a.radius;
    } else if (a.type == MLX_OBSTACLE_BOX) {
      for (int r = 0; r < 3; ++r) {
        const double* row = a.rotation + 3 * r;
        const double nr = std::sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2]);
        if (!(nr > 0)) return set_error(MLX_ERR_ARGUMENT, "box rotation has a zero row");
        for (int d = 0; d < 3; ++d) o.dir[3 * r + d] = row[d] / nr;
        o.half[r] = a.scale[r] / 2;
      }
    } else {
      return set_error(MLX_ERR_ARGUMENT, "unknown obstacle type");
    }
    out.push_back(o);
  }
  return MLX_OK;
}

// Masks and the ordered list of contact vertices of positions x0 (stream
// work only).  Uses d_obs / sim_obs.
template <typename R>
int Solver<R>::detect_contacts(const R4<R>* x0) {
  const int nb = blocks_for(N, 256);
  const int nobs = (int)sim_obs.size();
  k_contact_mask<R><<<nb, 256, 0, stream>>>(x0, N, d_obs.as<Obstacle>(), nobs, d_cmask.as<unsigned>());
  int* scan = d_cscan.as<int>();
  k_compact_count<<<nb, 256, 0, stream>>>(d_cmask.as<unsigned>(), N, -1, scan);
  k_compact_scan<<<1, 1024, 0, stream>>>(scan, nb, nullptr, scan + nb);
  k_compact_scatter<<<nb, 256, 0, stream>>>(d_cmask.as<unsigned>(), N, -1, scan, d_cverts.as<int>(),
                                            d_cidx.as<int>());
  // finder list lengths (the residual's K x K expansion counts them)
  CU(cudaMemsetAsync(scan + nb + 2, 0, sizeof(int) * nobs, stream));
  k_obstacle_counts<<<std::min(nb, 296), 256, 0, stream>>>(d_cmask.as<unsigned>(), N, nobs, scan + nb + 2);
  CU(cudaGetLastError());
  if (sim.P.contact_coloring) {
    const DevContacts dc = dev_contacts();
    CU(cudaMemsetAsync(d_chist.p, 0, sizeof(int) * (size_t)(C + 1), stream));
    k_cc_hist<<<nb, 256, 0, stream>>>(dc, d_chist.as<int>());
    k_cc_offsets<<<1, 32, 0, stream>>>(d_chist.as<int>(), C + 1, d_coff.as<int>(), d_ccur.as<int>());
    k_cc_scatter<<<nb, 256, 0, stream>>>(dc, d_ccur.as<int>(), d_cbucket.as<int>());
    CU(cudaGetLastError());
  }
  return MLX_OK;
}

// contact_coloring: the colour phase of each vertex's elastic contacts is the
// first colour none of the vertex's tets has (C when every colour does), and
// the buffers of the per-step buckets.
template <typename R>
int Solver<R>::contact_colours() {
  if (d_vcc.p) return MLX_OK;
  const int words = (C + 64) / 64;
  std::vector<uint64_t> used((size_t)N * words, 0);
  for (int c = 0; c < C; ++c)
    for (int s = color_off[c]; s < color_off[c + 1]; ++s) {
      const int4 v = vid_sorted[s];
      for (int k : {v.x, v.y, v.z, v.w}) used[(size_t)k * words + c / 64] |= 1ull << (c % 64);
    }
  std::vector<int> vcc(N, C);
  for (int v = 0; v < N; ++v)
    for (int c = 0; c < C; ++c)
      if (!((used[(size_t)v * words + c / 64] >> (c % 64)) & 1ull)) {
        vcc[v] = c;
        break;
      }
  CHECK(d_vcc.ensure(sizeof(int) * (size_t)N));
  CHECK(d_cbucket.ensure(sizeof(int) * (size_t)N));
  CHECK(d_coff.ensure(sizeof(int) * (size_t)(C + 2)));
  CHECK(d_ccur.ensure(sizeof(int) * (size_t)(C + 1)));
  CHECK(d_chist.ensure(sizeof(int) * (size_t)(C + 1)));
  CU(cudaMemcpyAsync(d_vcc.p, vcc.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice, stream));
  CU(cudaMemsetAsync(d_coff.p, 0, sizeof(int) * (size_t)(C + 2), stream));
  CU(cudaStreamSynchronize(stream));
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_set_obstacles(const mlx_obstacle* obs, int nobs, double restitution) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "mlx_sim_init first");
  std::vector<Obstacle> o;
  CHECK(prepare_obstacles(obs, nobs, o));
  DeviceGuard g(device);
  sim_obs = o;
  sim_restitution = restitution;
  if (!o.empty()) {
    CHECK(d_obs.ensure(sizeof(Obstacle) * o.size()));
    CHECK(d_cmask.ensure(sizeof(unsigned) * N));
    CHECK(d_cverts.ensure(sizeof(int) * N));
    CHECK(d_cidx.ensure(sizeof(int) * N));
    CHECK(d_cscan.ensure(sizeof(int) * (blocks_for(N, 256) + 2 + MLX_MAX_OBSTACLES)));
    CHECK(d_clam_dev.ensure(sizeof(double) * (size_t)N * o.size()));
    CU(cudaMemcpyAsync(d_obs.p, o.data(), sizeof(Obstacle) * o.size(), cudaMemcpyHostToDevice, stream));
    CHECK(contact_colours());
    CU(cudaMemsetAsync(d_cscan.p, 0, sizeof(int) * (blocks_for(N, 256) + 2 + MLX_MAX_OBSTACLES), stream));
    CU(cudaStreamSynchronize(stream));
  }
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_monitor(double* ra, int cap, int32_t* len, int32_t* total_it, double* run_until, int32_t* status) {
  if (!sim_last.valid) return set_error(MLX_ERR_ARGUMENT, "no monitored step has run (compute_residuals = 0?)");
  int n = 0, tot = 0, err = 0;
  double ru = sim.P.run_until;
  std::vector<double> r;
  if (sim_last.device) {
    DeviceGuard g(device);
    MonState hdr;
    const size_t head = offsetof(MonState, ra);
    CU(cudaMemcpyAsync(&hdr, d_mon.p, head, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    n = hdr.ra_len;
    tot = hdr.total_iterations;
    err = hdr.error;
    ru = hdr.run_until;
    r.resize(n);
    if (n) CU(cudaMemcpyAsync(r.data(), mon()->ra, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
  } else {
    r = sim_last.ra;
    n = (int)r.size();
    tot = sim_last.total_it;
  }
  if (len) *len = n;
  if (total_it) *total_it = tot;
  if (run_until) *run_until = ru;
  if (status) *status = err;
  if (ra && cap > 0) std::memcpy(ra, r.data(), sizeof(double) * std::min(cap, n));
  return MLX_OK;
}

// Multiplier warm start of the resident stepper: on = 1 starts the last
// layer of every step from a lambda_{n-1} + b (lambda_{n-1} - lambda_{n-2});
// every call forgets the steps saved so far.
template <typename R>
int Solver<R>::mws_configure(int on, double a, double b) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "mlx_sim_init first");
  if (!std::isfinite(a) || !std::isfinite(b)) return set_error(MLX_ERR_ARGUMENT, "coefficients must be finite");
  DeviceGuard g(device);
  mws.on = on ? 1 : 0;
  mws.a = a;
  mws.b = b;
  mws.rows = mat_kind == MAT_NH ? 2 : 6;
  if (mws.on) {
    const size_t bytes = sizeof(R) * (size_t)mws.rows * T;
    CHECK(mws.d_lam1.ensure(bytes));
    CHECK(mws.d_lam2.ensure(bytes));
    CHECK(mws.d_seen.ensure(sizeof(int)));
    CU(cudaMemsetAsync(mws.d_lam1.p, 0, bytes, stream));
    CU(cudaMemsetAsync(mws.d_lam2.p, 0, bytes, stream));
    CU(cudaMemsetAsync(mws.d_seen.p, 0, sizeof(int), stream));
    CU(cudaStreamSynchronize(stream));
  }
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  return MLX_OK;
}

// Starting multipliers of the last layer and the position shift they imply
// (after the layer's elastic release, before its projectGS loop).
template <typename R>
int Solver<R>::mws_start() {
  TetData<R> td = tets();
  for (int c = 0; c < C; ++c) {
    const int begin = color_off[c], count = color_off[c + 1] - color_off[c];
    if (count <= 0) continue;
    if (mat_kind == MAT_NH)
      k_ws_lambda_shift<R, MAT_NH><<<blocks_for(count, 256), 256, 0, stream>>>(
          td, begin, count, pos(), d_pin_mask.as<unsigned char>(), mws.d_lam1.as<R>(), mws.d_lam2.as<R>(), mws.a,
          mws.b, mws.d_seen.as<int>());
    else
      k_ws_lambda_shift<R, MAT_STVK_LAME><<<blocks_for(count, 256), 256, 0, stream>>>(
          td, begin, count, pos(), d_pin_mask.as<unsigned char>(), mws.d_lam1.as<R>(), mws.d_lam2.as<R>(), mws.a,
          mws.b, mws.d_seen.as<int>());
    CU(cudaGetLastError());
  }
  return MLX_OK;
}

template <typename R>
int Solver<R>::ws_after_make_rigids(const LayerWork& w) {
  const int nb = ws.nb;
  k_ws_own<R><<<nb, 256, 0, stream>>>(ws.S, w.bodies.as<Body>(), pos(), ws.d_own.as<float>(), ws.d_rec.as<double>());
  const float* nrm = ws.d_norm.as<float>();
  const float* om = nrm + 2 * kWsFeat;
  const float* os = om + kWsOut;
  k_ws_features<<<blocks_for(nb, 128), 128, 0, stream>>>(ws.S, ws.d_own.as<float>(), nrm, nrm + kWsFeat,
                                                         ws.d_raw.as<float>(),
                                                         ws.mode == 1 ? ws.d_feat.as<float>() : nullptr);
  CU(cudaGetLastError());
  if (ws.mode == 0) return MLX_OK;
  if (ws.mode == 1) {
    CHECK(mlp_forward_on_stream(ws.net, ws.d_feat.as<float>(), nb, stream, &ws.y, &ws.ld));
  } else {
    ws.y = ws.d_corr.as<float>();
    ws.ld = kWsOut;
  }
  CU(cudaMemsetAsync(ws.d_fallback.p, 0, sizeof(int), stream));
  k_ws_apply_velocity<<<blocks_for(nb, 128), 128, 0, stream>>>(nb, w.bodies.as<Body>(), ws.y, ws.ld, om, os,
                                                               ws.gate, ws.d_fallback.as<int>());
  CU(cudaGetLastError());
  return MLX_OK;
}

template <typename R>
int Solver<R>::ws_after_lamb_reset(const LayerWork& w) {
  const float* om = ws.d_norm.as<float>() + 2 * kWsFeat;
  k_ws_apply_lambda<<<ws.nb, 128, 0, stream>>>(ws.S, w.lamB.as<double>(), ws.y, ws.ld, om, om + kWsOut, ws.gate);
  CU(cudaGetLastError());
  return MLX_OK;
}

// Sets up the warm start on the first layer of the resident stepper (its
// rigid clusters): rest data and nearest neighbours of the clusters, the
// normalisation of features (mean, std: 44 each) and outputs (8 each), the
// perceptron (mode 1) or fixed corrections (mode 2, clusters x 8 in output
// units), and whether every step keeps its features and targets.
template <typename R>
int Solver<R>::ws_configure(int record, int mode, mlx_mlp* net, double gate, const float* fmean, const float* fstd,
                            const float* omean, const float* ostd, const float* corrections, int32_t* nb_out) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "mlx_sim_init first");
  if (mode < 0 || mode > 2) return set_error(MLX_ERR_ARGUMENT, "warm start mode must be 0, 1 or 2");
  DeviceGuard g(device);
  const int col = sim.ld.num_layers > 0 ? sim.ld.layers_map[0] - 1 : -1;
  if (col < 0 || sim_work.cache.size() <= (size_t)col || sim_work.cache[col]->nb == 0)
    return set_error(MLX_ERR_ARGUMENT, "the first layer has no rigid clusters to warm-start");
  LayerStatic& ls = *sim_work.cache[col];
  const int nb = ls.nb;
  if (mode == 1) {
    int ni = 0, no = 0, mb = 0;
    CHECK(mlp_dims(net, &ni, &no, &mb));
    if (ni != kWsFeat || no != kWsOut || mb < nb)
      return set_error(MLX_ERR_ARGUMENT, "the perceptron must map 44 features to 8 outputs for every cluster");
    if (!fmean || !fstd || !omean || !ostd) return set_error(MLX_ERR_ARGUMENT, "normalisation arrays are NULL");
  }
  if (mode == 2 && !corrections) return set_error(MLX_ERR_ARGUMENT, "corrections are NULL");
  if (std::isnan(gate)) return set_error(MLX_ERR_ARGUMENT, "the fallback gate is NaN");
  ws.reset();
  // rest positions and per-cluster rest data
  std::vector<double4> rest(N);
  for (int v = 0; v < N; ++v) rest[v] = make_double4(sim_p0[3 * v], sim_p0[3 * v + 1], sim_p0[3 * v + 2], 0);
  CHECK(ws.d_rest.ensure(sizeof(double4) * N));
  CU(cudaMemcpyAsync(ws.d_rest.p, rest.data(), sizeof(double4) * N, cudaMemcpyHostToDevice, stream));
  // d_static: nbr int[nb*4] | rest_com[nb*3] | rest_cinv[nb*9] | mass[nb]
  const size_t o_com = ((size_t)nb * kWsNbr * sizeof(int) + 15) / 16 * 16;
  const size_t o_cinv = o_com + sizeof(double) * 3 * nb, o_mass = o_cinv + sizeof(double) * 9 * nb;
  CHECK(ws.d_static.ensure(o_mass + sizeof(double) * nb));
  char* base = static_cast<char*>(ws.d_static.p);
  const int* dint = ls.dev.as<int>();
  WsStatic S{};
  S.nb = nb;
  S.body_vert_off = dint + ls.o_bvo;
  S.body_verts = dint + ls.o_bv;
  S.bnd_off = dint + ls.o_bo;
  S.nbr = reinterpret_cast<const int*>(base);
  S.rest_com = reinterpret_cast<const double*>(base + o_com);
  S.rest_cinv = reinterpret_cast<const double*>(base + o_cinv);
  S.mass = reinterpret_cast<const double*>(base + o_mass);
  S.rest = ws.d_rest.as<double4>();
  S.vmass = d_vmass.as<double>();
  k_ws_rest<<<nb, 256, 0, stream>>>(S, reinterpret_cast<double*>(base + o_com),
                                    reinterpret_cast<double*>(base + o_cinv), reinterpret_cast<double*>(base + o_mass));
  CU(cudaGetLastError());
  std::vector<double> com(3 * (size_t)nb);
  CU(cudaMemcpyAsync(com.data(), base + o_com, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  // the kWsNbr clusters nearest at rest (ties: lower index)
  std::vector<int> nbr((size_t)nb * kWsNbr, -1);
  std::vector<std::pair<double, int>> d;
  for (int b = 0; b < nb; ++b) {
    d.clear();
    for (int c = 0; c < nb; ++c) {
      if (c == b) continue;
      const double dx = com[3 * c] - com[3 * b], dy = com[3 * c + 1] - com[3 * b + 1], dz = com[3 * c + 2] - com[3 * b + 2];
      d.emplace_back(dx * dx + dy * dy + dz * dz, c);
    }
    const size_t k = std::min<size_t>(kWsNbr, d.size());
    std::partial_sort(d.begin(), d.begin() + k, d.end());
    for (size_t q = 0; q < k; ++q) nbr[(size_t)b * kWsNbr + q] = d[q].second;
  }
  CU(cudaMemcpyAsync(base, nbr.data(), sizeof(int) * nbr.size(), cudaMemcpyHostToDevice, stream));
  // normalisation: fmean | fstd | omean | ostd (identity when not given)
  std::vector<float> nrm(2 * kWsFeat + 2 * kWsOut);
  for (int i = 0; i < kWsFeat; ++i) {
    nrm[i] = fmean ? fmean[i] : 0.f;
    nrm[kWsFeat + i] = fstd ? fstd[i] : 1.f;
  }
  for (int i = 0; i < kWsOut; ++i) {
    nrm[2 * kWsFeat + i] = (mode == 1 && omean) ? omean[i] : 0.f;
    nrm[2 * kWsFeat + kWsOut + i] = (mode == 1 && ostd) ? ostd[i] : 1.f;
  }
  CHECK(ws.d_norm.ensure(sizeof(float) * nrm.size()));
  CU(cudaMemcpyAsync(ws.d_norm.p, nrm.data(), sizeof(float) * nrm.size(), cudaMemcpyHostToDevice, stream));
  CHECK(ws.d_own.ensure(sizeof(float) * kWsOwn * nb));
  CHECK(ws.d_raw.ensure(sizeof(float) * kWsFeat * nb));
  CHECK(ws.d_feat.ensure(sizeof(float) * kWsFeat * nb));
  CHECK(ws.d_rec.ensure(sizeof(double) * kWsRec * nb));
  CHECK(ws.d_target.ensure(sizeof(float) * kWsOut * nb));
  CHECK(ws.d_corr.ensure(sizeof(float) * kWsOut * nb));
  CHECK(ws.d_fallback.ensure(sizeof(int)));
  CU(cudaMemsetAsync(ws.d_fallback.p, 0, sizeof(int), stream));
  CU(cudaMemsetAsync(ws.d_target.p, 0, sizeof(float) * kWsOut * nb, stream));
  if (mode == 2)
    CU(cudaMemcpyAsync(ws.d_corr.p, corrections, sizeof(float) * kWsOut * nb, cudaMemcpyHostToDevice, stream));
  CU(cudaStreamSynchronize(stream));
  ws.S = S;
  ws.record = record;
  ws.mode = mode;
  ws.gate = gate;
  ws.net = net;
  ws.col = col;
  ws.nb = nb;
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  if (nb_out) *nb_out = nb;
  return MLX_OK;
}

template <typename R>
int Solver<R>::ws_fetch(float* features, float* targets, int cap, int32_t* nb, int32_t* fallbacks) {
  if (ws.nb == 0) return set_error(MLX_ERR_ARGUMENT, "warm start not configured");
  if (nb) *nb = ws.nb;
  if (cap < ws.nb) return set_error(MLX_ERR_LIMIT, "capacity below the number of clusters");
  DeviceGuard g(device);
  if (features)
    CU(cudaMemcpyAsync(features, ws.d_raw.p, sizeof(float) * kWsFeat * ws.nb, cudaMemcpyDeviceToHost, stream));
  if (targets)
    CU(cudaMemcpyAsync(targets, ws.d_target.p, sizeof(float) * kWsOut * ws.nb, cudaMemcpyDeviceToHost, stream));
  int fb = 0;
  if (fallbacks && ws.d_fallback.p)
    CU(cudaMemcpyAsync(&fb, ws.d_fallback.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  if (fallbacks) *fallbacks = fb;
  return MLX_OK;
}

template <typename R>
int Solver<R>::pcg_setup() {
  if (pcg_ready) return MLX_OK;
  if (pcg_vol.empty()) return set_error(MLX_ERR_UNSUPPORTED, "the PCG system needs mu and lambda in the mesh description");
  CHECK(vt_setup());
  CHECK(d_pcg_G.ensure(sizeof(double) * pcg_G.size()));
  CHECK(d_pcg_vol.ensure(sizeof(double) * T));
  CHECK(d_pcg_lame.ensure(sizeof(double) * 2 * (size_t)T));
  CU(cudaMemcpyAsync(d_pcg_G.p, pcg_G.data(), sizeof(double) * pcg_G.size(), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_pcg_vol.p, pcg_vol.data(), sizeof(double) * T, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_pcg_lame.p, pcg_lame.data(), sizeof(double) * 2 * (size_t)T, cudaMemcpyHostToDevice, stream));
  CU(cudaStreamSynchronize(stream));
  pcg_ready = true;
  return MLX_OK;
}

// The vertex -> (tet, corner) CSR of the matrix-free operators (fixed order:
// sorted tet id, then corner), the pinned-DOF mask and the PCG's vectors.
template <typename R>
int Solver<R>::vt_setup() {
  if (vt_ready) return MLX_OK;
  std::vector<int> off(N + 1, 0);
  for (int sidx = 0; sidx < T; ++sidx) {
    const int4 q = vid_sorted[sidx];
    for (int v : {q.x, q.y, q.z, q.w}) ++off[v + 1];
  }
  for (int v = 0; v < N; ++v) off[v + 1] += off[v];
  std::vector<int2> vt(off[N]);
  std::vector<int> vtpos(4 * (size_t)T);
  {
    std::vector<int> f(off.begin(), off.end() - 1);
    for (int sidx = 0; sidx < T; ++sidx) {
      const int4 q = vid_sorted[sidx];
      const int vv[4] = {q.x, q.y, q.z, q.w};
      for (int k = 0; k < 4; ++k) {
        vtpos[4 * (size_t)sidx + k] = f[vv[k]];
        vt[f[vv[k]]++] = make_int2(sidx, k);
      }
    }
  }
  CHECK(d_vtpos.ensure(sizeof(int) * vtpos.size()));
  CU(cudaMemcpyAsync(d_vtpos.p, vtpos.data(), sizeof(int) * vtpos.size(), cudaMemcpyHostToDevice, stream));
  std::vector<unsigned char> pm(N, 0);
  for (int d : pinned) pm[d / 3] |= (unsigned char)(1u << (d % 3));
  CHECK(d_pcg_vt.ensure(sizeof(int) * (N + 1) + sizeof(int2) * vt.size()));
  CHECK(d_pcg_pin.ensure(N));
  // CSR: vt pairs first (8-byte aligned), then the offsets
  CU(cudaMemcpyAsync(d_pcg_vt.p, vt.data(), sizeof(int2) * vt.size(), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(static_cast<char*>(d_pcg_vt.p) + sizeof(int2) * vt.size(), off.data(), sizeof(int) * (N + 1),
                     cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_pcg_pin.p, pm.data(), N, cudaMemcpyHostToDevice, stream));
  CHECK(d_pcg_vec.ensure(sizeof(double4) * 7 * (size_t)N));
  CHECK(d_pcg_P.ensure(sizeof(double) * 9 * (size_t)N));
  CHECK(d_pcg_part.ensure(sizeof(double) * 4 * 296));  // two sets of partials
  CHECK(d_pcg_sc.ensure(sizeof(PcgScalars)));
  CU(cudaStreamSynchronize(stream));
  vt_ready = true;
  return MLX_OK;
}

// The rows of the assembled J^T W J (pcg.cuh k_ns_assemble): for every
// vertex the vertices sharing a tet with it, in increasing order, and for
// every pair of the vertex CSR the row slots of its tet's four corners.
// Fixed by the mesh, built once.
template <typename R>
int Solver<R>::ns_topology() {
  if (d_ns_K.p) return MLX_OK;
  std::vector<int> off(N + 1, 0);
  for (int sidx = 0; sidx < T; ++sidx) {
    const int4 q = vid_sorted[sidx];
    for (int v : {q.x, q.y, q.z, q.w}) ++off[v + 1];
  }
  for (int v = 0; v < N; ++v) off[v + 1] += off[v];
  std::vector<int> pt(off[N]);  // the vertex CSR's tets, in the order vt_setup stores them
  {
    std::vector<int> f(off.begin(), off.end() - 1);
    for (int sidx = 0; sidx < T; ++sidx) {
      const int4 q = vid_sorted[sidx];
      for (int v : {q.x, q.y, q.z, q.w}) pt[f[v]++] = sidx;
    }
  }
  std::vector<int> nb_off(N + 1, 0), nb_col;
  std::vector<unsigned int> pslot(off[N]);
  nb_col.reserve((size_t)N * 16);
  std::vector<int> row;
  for (int v = 0; v < N; ++v) {
    row.clear();
    for (int k = off[v]; k < off[v + 1]; ++k) {
      const int4 q = vid_sorted[pt[k]];
      row.insert(row.end(), {q.x, q.y, q.z, q.w});
    }
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    if (row.size() > 255)
      return set_error(MLX_ERR_UNSUPPORTED, "a vertex shares tets with more than 254 other vertices");
    for (int k = off[v]; k < off[v + 1]; ++k) {
      const int4 q = vid_sorted[pt[k]];
      unsigned int sl = 0;
      int b = 0;
      for (int c : {q.x, q.y, q.z, q.w})
        sl |= (unsigned int)(std::lower_bound(row.begin(), row.end(), c) - row.begin()) << (8 * b++);
      pslot[k] = sl;
    }
    nb_col.insert(nb_col.end(), row.begin(), row.end());
    nb_off[v + 1] = (int)nb_col.size();
  }
  CHECK(d_ns_nb.ensure(sizeof(int) * (N + 1 + nb_col.size())));
  CHECK(d_ns_pslot.ensure(sizeof(unsigned int) * pslot.size()));
  CHECK(d_ns_K.ensure(sizeof(R) * 9 * nb_col.size()));
  CU(cudaMemcpyAsync(d_ns_nb.p, nb_off.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(d_ns_nb.as<int>() + N + 1, nb_col.data(), sizeof(int) * nb_col.size(), cudaMemcpyHostToDevice,
                     stream));
  CU(cudaMemcpyAsync(d_ns_pslot.p, pslot.data(), sizeof(unsigned int) * pslot.size(), cudaMemcpyHostToDevice,
                     stream));
  CU(cudaStreamSynchronize(stream));
  return MLX_OK;
}

template <typename R>
NsBlocks Solver<R>::ns_blocks() const {
  NsBlocks b;
  b.nb_off = d_ns_nb.as<int>();
  b.nb_col = d_ns_nb.as<int>() + N + 1;
  b.pslot = d_ns_pslot.as<unsigned int>();
  b.vtpos = d_vtpos.as<int>();
  return b;
}

template <typename R>
PcgOp Solver<R>::vt_op(double h2) {
  const size_t npairs = (d_pcg_vt.bytes - sizeof(int) * (N + 1)) / sizeof(int2);
  PcgOp op;
  op.N = N;
  op.vt = d_pcg_vt.as<int2>();
  op.vt_off = reinterpret_cast<const int*>(static_cast<const char*>(d_pcg_vt.p) + sizeof(int2) * npairs);
  op.vid = d_vid.as<int4>();
  op.G = d_pcg_G.as<double>();
  op.vol = d_pcg_vol.as<double>();
  op.lame = d_pcg_lame.as<double>();
  op.vmass = d_vmass.as<double>();
  op.pin = d_pcg_pin.as<unsigned char>();
  op.h2 = h2;
  return op;
}

// The PCG in the layer solve of a Neo-Hookean mesh: `pcg_iterations` PCG
// iterations per Newton correction of the last layer (0 turns it off),
// before its Gauss-Seidel and after every `every` of its iterations (0: only
// before).  Set-up (buffers, the vertex CSR) happens here, outside any
// capture; cached step graphs are dropped.
template <typename R>
int Solver<R>::ns_configure(int pcg_iterations, int every) {
  if (pcg_iterations < 0 || every < 0) return set_error(MLX_ERR_ARGUMENT, "iterations and interval must be >= 0");
  if (pcg_iterations > 0 && mat_kind != MAT_NH)
    return set_error(MLX_ERR_UNSUPPORTED, "the layer PCG covers the Neo-Hookean constraint pair");
  DeviceGuard g(device);
  if (pcg_iterations > 0) {
    CHECK(vt_setup());
    CHECK(ns_topology());
    CHECK(d_ns_jac.ensure(sizeof(R) * 48 * (size_t)T));      // tet-major and CSR-order copies
    CHECK(d_ns_tet.ensure(sizeof(double2) * 3 * (size_t)T));  // w, c, q
    CHECK(d_pcg_part.ensure(sizeof(double) * 2 * kNsMaxPartials));
    // the vertex pass's grid: the blocks resident at once, at most one
    // partial sum each
    int per_sm = 0, sms = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ns_spmv<R>, 256, 0));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    ns_vertex_blocks = std::max(1, std::min(per_sm * sms, kNsMaxPartials));
  }
  ns_iters = pcg_iterations;
  ns_every = every;
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  drop_host_graph();
  return MLX_OK;
}

// One Newton-PCG correction of the current positions and multipliers
// (pcg.cuh): stream work only, so it can be captured.
template <typename R>
int Solver<R>::ns_correct(double h, long long* launches) {
  const PcgOp op = vt_op(h * h);
  const int nb = blocks_for(N, 256), tb = blocks_for(T, 256), nred = std::min(nb, 296);
  R* jt = d_ns_jac.as<R>();
  R* jv = jt + (size_t)24 * T;
  double2* tw = d_ns_tet.as<double2>();
  double2 *w = tw, *c = tw + T, *q = tw + 2 * (size_t)T;
  double4* V = d_pcg_vec.as<double4>();
  double4 *db = V, *dx = V + N, *dr = V + 2 * (size_t)N, *dz = V + 3 * (size_t)N, *dd = V + 4 * (size_t)N,
          *dAp = V + 5 * (size_t)N;
  double* P = d_pcg_P.as<double>();
  double* part = d_pcg_part.as<double>();
  PcgScalars* sc = d_pcg_sc.as<PcgScalars>();
  const int4* vid = d_vid.as<int4>();
  k_ns_jacobian<R><<<tb, 256, 0, stream>>>(tets(), pos(), h * h, d_vtpos.as<int>(), jt, jv, w, c, q);
  k_ns_rhs<R><<<blocks_for((long long)N * kNsTeam, 256), 256, 0, stream>>>(op, jv, q, db);  // b = -J^T (W C + lambda)
  CU(cudaMemsetAsync(dx, 0, sizeof(double4) * N, stream));
  CU(cudaMemcpyAsync(dr, db, sizeof(double4) * N, cudaMemcpyDeviceToDevice, stream));
  const NsBlocks nbk = ns_blocks();
  R* K = d_ns_K.as<R>();
  k_ns_assemble<R><<<blocks_for(N, kNsAsmWarps), 32 * kNsAsmWarps, 0, stream>>>(op, nbk, jv, w, K, P);  // K, P
  k_pcg_precond<<<nb, 256, 0, stream>>>(N, P, op.pin, dr, dz);
  // beta = 0, d = 0 (the first direction is z) and the last-block counts 0;
  // then rTz = r'z of the start
  CU(cudaMemsetAsync(dd, 0, sizeof(double4) * N, stream));
  CU(cudaMemsetAsync(sc, 0, sizeof(PcgScalars), stream));
  k_pcg_dot2<<<nred, 256, 0, stream>>>(N, dr, dz, nullptr, nullptr, part);
  k_pcg_scalars<<<1, 256, 0, stream>>>(part, nred, 0, sc, nullptr, 0);
  const int vb = std::max(1, std::min(blocks_for((long long)N * kNsTeam, 256), ns_vertex_blocks));
  double* part2 = part + kNsMaxPartials;
  double4* D[2] = {dd, V + 6 * (size_t)N};  // the direction, alternating
  for (int i = 0; i < ns_iters; ++i) {
    k_ns_spmv<R><<<vb, 256, 0, stream>>>(op, nbk, K, dz, D[i & 1], D[(i + 1) & 1], dAp, sc, part,
                                         &sc->count[0]);  // d, Ap = A d, alpha
    k_ns_step<<<nred, 256, 0, stream>>>(N, sc, D[(i + 1) & 1], dAp, dx, dr, P, op.pin, dz, part2,
                                        &sc->count[1]);  // x, r, z, beta
  }
  k_ns_lambda<R><<<tb, 256, 0, stream>>>(T, vid, jt, w, c, dx, d_lambda.as<R>());
  k_ns_move<R><<<nb, 256, 0, stream>>>(N, dx, pos());
  CU(cudaGetLastError());
  if (launches) *launches += 7 + 2LL * ns_iters;
  return MLX_OK;
}

// solvePCG (2d/tools/solver/solvePCG.m) with x0 = 0 for A = M + h^2 K0 on
// the unpinned DOFs and the block-Jacobi preconditioner (pcg.cuh).  The
// iteration runs as stream work only; alpha and beta stay on the device.
template <typename R>
int Solver<R>::pcg_solve(double h, const double* b, int iterations, double* x, double* resvec) {
  if (!b || !x) return set_error(MLX_ERR_ARGUMENT, "null argument");
  if (iterations < 0 || !(h > 0)) return set_error(MLX_ERR_ARGUMENT, "need iterations >= 0 and h > 0");
  DeviceGuard g(device);
  CHECK(pcg_setup());
  const PcgOp op = vt_op(h * h);
  double4* V = d_pcg_vec.as<double4>();
  double4 *db = V, *dx = V + N, *dr = V + 2 * (size_t)N, *dz = V + 3 * (size_t)N, *dd = V + 4 * (size_t)N,
          *dAp = V + 5 * (size_t)N, *dtmp = V + 6 * (size_t)N;
  double* P = d_pcg_P.as<double>();
  double* part = d_pcg_part.as<double>();
  PcgScalars* sc = d_pcg_sc.as<PcgScalars>();
  CHECK(d_pcg_res.ensure(sizeof(double) * std::max(iterations, 1)));
  double* dres = resvec ? d_pcg_res.as<double>() : nullptr;
  const int nb = blocks_for(N, 256), nred = std::min(nb, 296);
  CHECK(d_stage.ensure(sizeof(double) * 3 * (size_t)N));
  CU(cudaMemcpyAsync(d_stage.p, b, sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice, stream));
  k_load_vec<double><<<nb, 256, 0, stream>>>(d_stage.as<double>(), dtmp, N);
  k_pcg_mask<<<nb, 256, 0, stream>>>(N, op.pin, dtmp, db);               // b on the unpinned DOFs
  CU(cudaMemsetAsync(dx, 0, sizeof(double4) * N, stream));               // x = x0 = 0
  CU(cudaMemcpyAsync(dr, db, sizeof(double4) * N, cudaMemcpyDeviceToDevice, stream));  // r = b - A x0
  k_pcg_block_jacobi<<<nb, 256, 0, stream>>>(op, P);
  k_pcg_precond<<<nb, 256, 0, stream>>>(N, P, op.pin, dr, dz);           // z = P r
  CU(cudaMemcpyAsync(dd, dz, sizeof(double4) * N, cudaMemcpyDeviceToDevice, stream));  // d = z
  k_pcg_dot2<<<nred, 256, 0, stream>>>(N, dr, dz, nullptr, nullptr, part);
  k_pcg_scalars<<<1, 256, 0, stream>>>(part, nred, 0, sc, nullptr, 0);    // rTz = r'z
  for (int i = 0; i < iterations; ++i) {
    k_pcg_apply<<<nb, 256, 0, stream>>>(op, dd, dAp);                    // Ap = A d
    k_pcg_dot2<<<nred, 256, 0, stream>>>(N, dd, dAp, nullptr, nullptr, part);
    k_pcg_scalars<<<1, 256, 0, stream>>>(part, nred, 1, sc, nullptr, 0);  // alpha = rTz / d'Ap
    k_pcg_step<<<nb, 256, 0, stream>>>(N, sc, dd, dAp, dx, dr);         // x += alpha d, r -= alpha Ap
    k_pcg_precond<<<nb, 256, 0, stream>>>(N, P, op.pin, dr, dz);         // z = P r
    k_pcg_dot2<<<nred, 256, 0, stream>>>(N, dr, dz, nullptr, nullptr, part);
    k_pcg_scalars<<<1, 256, 0, stream>>>(part, nred, 2, sc, nullptr, 0);  // beta, rTz = r'z
    k_pcg_direction<<<nb, 256, 0, stream>>>(N, sc, dz, dd);              // d = z + beta d
    if (dres) {                                                          // resvec(i) = ||A x - b||
      k_pcg_apply<<<nb, 256, 0, stream>>>(op, dx, dAp);
      k_pcg_sub<<<nb, 256, 0, stream>>>(N, dAp, db, dtmp);
      k_pcg_dot2<<<nred, 256, 0, stream>>>(N, dtmp, dtmp, nullptr, nullptr, part);
      k_pcg_scalars<<<1, 256, 0, stream>>>(part, nred, 3, sc, dres, i);
      // the next iteration's A d overwrites dAp after this use
    }
  }
  CU(cudaGetLastError());
  k_store_pos<double><<<nb, 256, 0, stream>>>(dx, d_stage.as<double>(), N);
  CU(cudaMemcpyAsync(x, d_stage.p, sizeof(double) * 3 * (size_t)N, cudaMemcpyDeviceToHost, stream));
  if (resvec && iterations > 0)
    CU(cudaMemcpyAsync(resvec, dres, sizeof(double) * iterations, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_contact_count(int32_t* n) {
  if (!n) return set_error(MLX_ERR_ARGUMENT, "null argument");
  *n = 0;
  if (sim_obs.empty()) return MLX_OK;
  DeviceGuard g(device);
  CU(cudaMemcpyAsync(h_scalar.p, d_cscan.as<int>() + blocks_for(N, 256), sizeof(int), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  *n = h_scalar.as<int>()[0];
  return MLX_OK;
}

template <typename R>
int Solver<R>::find_contacts(const mlx_obstacle* obs, int nobs, const double* p, int max_contacts, int32_t* vids,
                             double* normals, double* points, double* comp, int32_t* K) {
  if (!p || !K) return set_error(MLX_ERR_ARGUMENT, "null argument");
  std::vector<Obstacle> o;
  CHECK(prepare_obstacles(obs, nobs, o));
  *K = 0;
  if (o.empty()) return MLX_OK;
  DeviceGuard g(device);
  const int nb = blocks_for(N, 256);
  const size_t cap = (size_t)N * o.size();
  DevBuf &dob = fc_ob, &dmask = fc_mask, &dverts = fc_verts, &dscan = fc_scan, &dx = fc_x, &dvid = fc_vid,
         &dout = fc_out, &dpos = fc_pos;
  CHECK(dob.ensure(sizeof(Obstacle) * o.size()));
  CHECK(dmask.ensure(sizeof(unsigned) * N));
  CHECK(dverts.ensure(sizeof(int) * cap));
  CHECK(dscan.ensure(sizeof(int) * (nb + o.size() + 1)));
  CHECK(dx.ensure(sizeof(double) * 3 * (size_t)N));
  CHECK(dpos.ensure(sizeof(double4) * N));
  CHECK(dvid.ensure(sizeof(int) * cap));
  CHECK(dout.ensure(sizeof(double) * 7 * cap));
  CU(cudaMemcpyAsync(dob.p, o.data(), sizeof(Obstacle) * o.size(), cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(dx.p, p, sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice, stream));
  CU(cudaMemsetAsync(dscan.p, 0, sizeof(int) * (nb + o.size() + 1), stream));
  // positions in FP64 whatever the solver's precision: detection on the caller's values
  k_load_pos<double><<<nb, 256, 0, stream>>>(dx.as<double>(), d_mass3.as<double>(), dpos.as<double4>(), N);
  const int no = (int)o.size();
  k_contact_mask<double><<<nb, 256, 0, stream>>>(dpos.as<double4>(), N, dob.as<Obstacle>(), no, dmask.as<unsigned>());
  int* blk = dscan.as<int>();
  int* tot = blk + nb;  // tot[f] = contacts before finder f
  double* out = dout.as<double>();
  for (int f = 0; f < no; ++f) {
    k_compact_count<<<nb, 256, 0, stream>>>(dmask.as<unsigned>(), N, f, blk);
    k_compact_scan<<<1, 1024, 0, stream>>>(blk, nb, tot + f, tot + f + 1);
    k_compact_scatter<<<nb, 256, 0, stream>>>(dmask.as<unsigned>(), N, f, blk, dverts.as<int>(), nullptr);
    k_contact_list<double><<<nb, 256, 0, stream>>>(dpos.as<double4>(), dob.as<Obstacle>(), f, dverts.as<int>(),
                                                   tot + f, tot + f + 1, (int)cap, dvid.as<int>(), out,
                                                   out + 3 * cap, out + 6 * cap);
  }
  CU(cudaGetLastError());
  int total = 0;
  CU(cudaMemcpyAsync(&total, tot + no, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  *K = total;
  if (total > max_contacts) return set_error(MLX_ERR_LIMIT, "more contacts than max_contacts");
  if (total == 0) return MLX_OK;
  if (!vids || !normals || !points || !comp) return set_error(MLX_ERR_ARGUMENT, "null output array");
  // the list's rows hold `total` entries each out of `cap`: copy those only
  CU(cudaMemcpyAsync(vids, dvid.p, sizeof(int) * total, cudaMemcpyDeviceToHost, stream));
  for (int d = 0; d < 3; ++d) {
    CU(cudaMemcpyAsync(normals + (size_t)d * total, out + (size_t)d * cap, sizeof(double) * total,
                       cudaMemcpyDeviceToHost, stream));
    CU(cudaMemcpyAsync(points + (size_t)d * total, out + (3 + (size_t)d) * cap, sizeof(double) * total,
                       cudaMemcpyDeviceToHost, stream));
  }
  CU(cudaMemcpyAsync(comp, out + 6 * cap, sizeof(double) * total, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  return MLX_OK;
}

template <typename R>
double Solver<R>::bytes_per_tet() const {
  // algorithmic bytes of one tet projection in this layout: vertex ids,
  // DmInv, volume, material, lambda read+write, four vertex records read and
  // written (+ four step-start records with Rayleigh damping)
  const double r = sizeof(R);
  const int nl = mat_kind == MAT_NH ? 2 : 6;
  const double vol = mat_kind == MAT_NH ? 0 : r;  // Neo-Hookean compliances include the volume
  double b = 16 + 9 * r + vol + mat_stride(mat_kind) * r + 2 * nl * r + 8 * 4 * r;
  if (damp) b += 4 * 4 * r;
  return b;
}

template <typename R>
double Solver<R>::group_bytes_per_tet() const {
  // the component-group path keeps the vertex records in shared memory: per
  // tet projection, corner slots, DmInv, volume, material and lambda read +
  // write (+ vertex ids and four step-start records with Rayleigh damping)
  const double r = sizeof(R);
  const int nl = mat_kind == MAT_NH ? 2 : 6;
  const double vol = mat_kind == MAT_NH ? 0 : r;
  double b = 16 + 9 * r + vol + mat_stride(mat_kind) * r + 2 * nl * r;
  if (damp) b += 16 + 4 * 4 * r;
  return b;
}

template <typename R>
int Solver<R>::record_event(cudaEvent_t e, bool capturing) {
  if (capturing) CU(cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal));
  else CU(cudaEventRecord(e, stream));
  return MLX_OK;
}

template <typename R>
int Solver<R>::enable_sweep_timing(int on) {
  DeviceGuard g(device);
  sweep_timing = on != 0;
  if (sim.graph) { cudaGraphExecDestroy(sim.graph); sim.graph = nullptr; }
  if (sweep_timing && tev.empty()) {
    long long pairs = 0;
    for (size_t l = 0; l < sim.iterations.size(); ++l) pairs += sim.iterations[l];
    pairs = std::max<long long>(pairs, 1);
    tev.resize(2 * pairs);
    for (cudaEvent_t& e : tev) CU(cudaEventCreate(&e));
    tev_bytes.assign(pairs, 0);
    tev_launches.assign(pairs, 0);
  }
  return MLX_OK;
}

template <typename R>
int Solver<R>::collect_sweep_times() {
  for (size_t q = 0; q + 1 < tev_used; q += 2) {
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, tev[q], tev[q + 1]));
    sweep_ms += ms;
    sweep_bytes += tev_bytes[q / 2];
    sweep_launches += tev_launches[q / 2];
  }
  return MLX_OK;
}

template <typename R>
int Solver<R>::sweep_stats(double* ms, double* bytes, long long* launches, int reset) {
  if (ms) *ms = sweep_ms;
  if (bytes) *bytes = sweep_bytes;
  if (launches) *launches = sweep_launches;
  if (reset) { sweep_ms = 0; sweep_bytes = 0; sweep_launches = 0; }
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_issue_step(long long* launches, bool capturing) {
  const double h = sim.P.h;
  tev_used = 0;
  R4<R>* p = pos();
  const bool devmon = capturing && sim.P.compute_residuals;
  if (devmon) {
    k_mon_step_begin<<<1, 1, 0, stream>>>(mon());
    CU(cudaGetLastError());
  }
  k_sim_begin<R><<<blocks_for(N, 256), 256, 0, stream>>>(p, d_vel.as<R4<R>>(), d_oldp.as<R4<R>>(),
                                                          d_resv.as<R4<R>>(), d_mass3.as<double>(),
                                                          d_pin_mask.as<unsigned char>(), N, h, sim.P.gravity,
                                                          sim.air_drag);
  CU(cudaGetLastError());
  CU(cudaMemsetAsync(d_lambda.p, 0, sizeof(R) * 6 * (size_t)T, stream));
  CHECK(reset_gsync());
  RunState st;
  st.runUntil = sim.P.run_until;
  st.residualArray.assign(1, 0.0);  // integrate's initialResidual (xpbdLayer3D.m:670-674)
  ContactData cd{};
  const DevContacts dc = dev_contacts();
  if (dc.nobs) {
    // contacts of the step-start positions (simulate3D detects on mesh3D.p
    // before integrate; oldp holds those positions now)
    CHECK(detect_contacts(d_oldp.as<R4<R>>()));
    st.launches += sim.P.contact_coloring ? 8 : 5;
  }
  CHECK(run_layers(&sim.ld, &sim.P, nullptr, cd, st, capturing, sim_work, dc));
  if (mws.on) {
    const long long n = (long long)mws.rows * T;
    k_ws_lambda_save<R><<<(int)((n + 255) / 256), 256, 0, stream>>>(n, d_lambda.as<R>(), mws.d_lam1.as<R>(),
                                                                   mws.d_lam2.as<R>(), mws.d_seen.as<int>());
    CU(cudaGetLastError());
    ++st.launches;
  }
  if (ws.nb > 0 && ws.record) {
    k_ws_targets<R><<<ws.nb, 256, 0, stream>>>(ws.S, p, d_oldp.as<R4<R>>(), ws.d_rec.as<double>(),
                                                sim_work.lamB.as<double>(), h, ws.d_target.as<float>());
    CU(cudaGetLastError());
    ++st.launches;
  }
  if (sim.P.compute_residuals) {
    sim_last.valid = true;
    sim_last.device = devmon;
    if (!devmon) {
      sim_last.ra = st.residualArray;
      sim_last.total_it = st.totalIterations;
      sim.P.run_until = st.runUntil;  // obj.runUntilResSmallerThan carries over to the next step
    }
  }
  k_sim_end<R><<<blocks_for(N, 256), 256, 0, stream>>>(p, d_oldp.as<R4<R>>(), d_vel.as<R4<R>>(), N, h);
  CU(cudaGetLastError());
  if (dc.nobs) {
    k_contact_velocity<R><<<blocks_for(N, 256), 256, 0, stream>>>(dc, d_oldp.as<R4<R>>(), d_vel.as<R4<R>>(), h,
                                                                  sim.P.gravity, sim_restitution);
    CU(cudaGetLastError());
    ++st.launches;
  }
  CU(cudaMemcpyAsync(h_gsync.p, d_gsync.p, sizeof(unsigned int) * 4, cudaMemcpyDeviceToHost, stream));
  if (launches) *launches = st.launches + 2;
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_step(int nsteps, int use_graph, double* device_ms) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "sim_setup has not been called");
  if (nsteps < 0) return set_error(MLX_ERR_ARGUMENT, "nsteps < 0");
  DeviceGuard g(device);
  if (use_graph && !sim.graph) {
    cudaGraph_t graph = nullptr;
    CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    long long nl = 0;
    int rc = sim_issue_step(&nl, true);
    cudaError_t e = cudaStreamEndCapture(stream, &graph);
    if (rc != MLX_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&sim.graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    sim.launches_per_step = nl;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (device_ms) {
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    CU(cudaEventRecord(e0, stream));
  }
  for (int s = 0; s < nsteps; ++s) {
    if (use_graph) {
      CU(cudaGraphLaunch(sim.graph, stream));
      if (sim.P.compute_residuals) {
        sim_last.valid = true;
        sim_last.device = true;
      }
    } else {
      long long nl = 0;
      // without a graph the residual monitor runs on the host
      CHECK(sim_issue_step(&nl, !sim.P.compute_residuals));
      sim.launches_per_step = nl;
    }
    if (sweep_timing) {  // the event pairs are reused by every step
      CU(cudaStreamSynchronize(stream));
      CHECK(collect_sweep_times());
      CHECK(check_gsync());
    }
  }
  if (device_ms) {
    CU(cudaEventRecord(e1, stream));
    CU(cudaEventSynchronize(e1));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    *device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  CU(cudaStreamSynchronize(stream));
  CHECK(check_gsync());
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_add_velocity(const int32_t* dofs, const double* dv, int n) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "sim_setup has not been called");
  if (n <= 0) return MLX_OK;
  std::vector<int> d0(n);
  for (int i = 0; i < n; ++i) {
    if (dofs[i] < 1 || dofs[i] > 3 * N) return set_error(MLX_ERR_ARGUMENT, "velocity DOF out of range");
    d0[i] = dofs[i] - 1;
  }
  DeviceGuard g(device);
  DevBuf dd, dvv;
  CHECK(dd.ensure(sizeof(int) * n));
  CHECK(dvv.ensure(sizeof(double) * n));
  CU(cudaMemcpyAsync(dd.p, d0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
  CU(cudaMemcpyAsync(dvv.p, dv, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  k_add_velocity<R><<<blocks_for(n, 256), 256, 0, stream>>>(d_vel.as<R4<R>>(), dd.as<int>(), dvv.as<double>(), n);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(stream));
  return MLX_OK;
}

template <typename R>
int Solver<R>::sim_get_state(double* p, double* v) {
  if (!sim.ready) return set_error(MLX_ERR_ARGUMENT, "sim_setup has not been called");
  DeviceGuard g(device);
  const size_t n3 = 3 * (size_t)N;
  CHECK(h_stage.ensure(sizeof(double) * 2 * n3));
  CHECK(d_stage.ensure(sizeof(double) * 2 * n3));
  double* ds = d_stage.as<double>();
  k_store_pos<R><<<blocks_for(N, 256), 256, 0, stream>>>(pos(), ds, N);
  k_store_pos<R><<<blocks_for(N, 256), 256, 0, stream>>>(d_vel.as<R4<R>>(), ds + n3, N);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(h_stage.p, ds, sizeof(double) * 2 * n3, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  if (p) std::memcpy(p, h_stage.p, sizeof(double) * n3);
  if (v) std::memcpy(v, h_stage.as<double>() + n3, sizeof(double) * n3);
  return MLX_OK;
}

template struct Solver<float>;
template struct Solver<double>;

SolverBase* make_solver(const mlx_mesh_desc* md, int* rc) {
  if (md->precision == MLX_FP64) {
    auto* s = new Solver<double>();
    *rc = s->create(md);
    return s;
  }
  auto* s = new Solver<float>();
  *rc = s->create(md);
  return s;
}

}  // namespace mlx

// ---------------------------------------------------------------------------
// C ABI
struct mlx_solver {
  int device;
  mlx::SolverBase* impl;
};

extern "C" {

const char* mlx_last_error(void) { return mlx::g_err.c_str(); }
int mlx_abi_version(void) { return MLX_ABI_VERSION; }

int mlx_device_count(void) {
  return mlx::guarded([&]() -> int {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    int good = 0;
    for (int d = 0; d < n; ++d) {
      cudaDeviceProp pr;
      if (cudaGetDeviceProperties(&pr, d) == cudaSuccess && pr.major == 10) ++good;
    }
    return good;
  });
}

int mlx_create(const mlx_mesh_desc* mesh, mlx_solver** out) {
  return mlx::guarded([&]() -> int {
    if (!mesh || !out) return set_error(MLX_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      return set_error(MLX_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (mesh->device < 0 || mesh->device >= n) return set_error(MLX_ERR_ARGUMENT, "device ordinal out of range");
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, mesh->device) != cudaSuccess || pr.major != 10)
      return set_error(MLX_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");
    int rc = MLX_OK;
    mlx::SolverBase* impl = mlx::make_solver(mesh, &rc);
    if (rc != MLX_OK) {
      delete impl;
      return rc;
    }
    *out = new mlx_solver{mesh->device, impl};
    return MLX_OK;
  });
}

int mlx_destroy(mlx_solver* s) {
  return mlx::guarded([&]() -> int {
    if (!s) return MLX_OK;
    {
      DeviceGuard g(s->device);
      delete s->impl;
    }
    delete s;
    return MLX_OK;
  });
}

int mlx_layer_solve(mlx_solver* s, const mlx_layer_desc* layers, const mlx_solve_params* params,
                    const mlx_contacts* contacts, const mlx_solve_inputs* in, mlx_solve_outputs* out) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->layer_solve(layers, params, contacts, in, out);
  });
}

int mlx_sim_init(mlx_solver* s, const mlx_layer_desc* layers, const mlx_solve_params* params, const double* p0,
                 const double* v0, double air_drag) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_init(layers, params, p0, v0, air_drag);
  });
}

int mlx_sim_add_velocity(mlx_solver* s, const int32_t* dofs, const double* dv, int32_t n) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    if (n > 0 && (!dofs || !dv)) return set_error(MLX_ERR_ARGUMENT, "null arrays");
    return s->impl->sim_add_velocity(dofs, dv, n);
  });
}

int mlx_sim_step(mlx_solver* s, int32_t nsteps, int32_t use_graph, double* device_ms) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_step(nsteps, use_graph, device_ms);
  });
}

int mlx_sim_get_state(mlx_solver* s, double* p, double* v) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_get_state(p, v);
  });
}

int mlx_sim_sweep_timing(mlx_solver* s, int32_t on) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->enable_sweep_timing(on);
  });
}

int mlx_sim_sweep_stats(mlx_solver* s, double* ms, double* bytes, long long* launches, int32_t reset) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sweep_stats(ms, bytes, launches, reset);
  });
}

long long mlx_sim_launches_per_step(const mlx_solver* s) { return s ? s->impl->sim_launches_per_step() : 0; }
long long mlx_last_call_launches(const mlx_solver* s) { return s ? s->impl->launches_last_call() : 0; }
int mlx_sim_autotune(mlx_solver* s, int32_t reps, double* before_ms, double* after_ms) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_autotune(reps, before_ms, after_ms);
  });
}
int mlx_find_contacts(mlx_solver* s, const mlx_obstacle* obstacles, int32_t num_obstacles, const double* p,
                      int32_t max_contacts, int32_t* vertex_ids, double* normals, double* point_colliders,
                      double* compliance, int32_t* num_contacts) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->find_contacts(obstacles, num_obstacles, p, max_contacts, vertex_ids, normals, point_colliders,
                                  compliance, num_contacts);
  });
}
int mlx_sim_set_obstacles(mlx_solver* s, const mlx_obstacle* obstacles, int32_t num_obstacles, double restitution) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_set_obstacles(obstacles, num_obstacles, restitution);
  });
}
int mlx_sim_monitor(mlx_solver* s, double* residuals, int32_t capacity, int32_t* len, int32_t* total_iterations,
                    double* run_until, int32_t* status) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_monitor(residuals, capacity, len, total_iterations, run_until, status);
  });
}
int mlx_sim_warm_start(mlx_solver* s, int32_t record, int32_t mode, mlx_mlp* net, double fallback_residual,
                       const float* feature_mean, const float* feature_std, const float* output_mean,
                       const float* output_std, const float* corrections, int32_t* num_clusters) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->ws_configure(record, mode, net, fallback_residual, feature_mean, feature_std, output_mean,
                                 output_std, corrections, num_clusters);
  });
}
int mlx_layer_pcg(mlx_solver* s, int32_t pcg_iterations, int32_t every) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->ns_configure(pcg_iterations, every);
  });
}
int mlx_sim_multiplier_warm_start(mlx_solver* s, int32_t on, double scale, double extrapolation) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->mws_configure(on, scale, extrapolation);
  });
}
int mlx_sim_warm_start_fetch(mlx_solver* s, float* features, float* targets, int32_t capacity, int32_t* num_clusters,
                             int32_t* num_fallbacks) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->ws_fetch(features, targets, capacity, num_clusters, num_fallbacks);
  });
}
int mlx_build_layers(mlx_solver* s, const double* p, const double* oldp, double h, int32_t ordering,
                     const int32_t* order, const double* DmInv, const double* sorted_layers, int32_t num_layers,
                     const uint8_t* forced_elastic, int32_t* rigid_body_sets, int32_t* num_rigids,
                     uint8_t* is_elastic_element, uint8_t* is_boundary_vertex, uint8_t* is_rigid_vertex,
                     int32_t* vertex_rigid_body) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->build_layers(p, oldp, h, ordering, order, DmInv, sorted_layers, num_layers, forced_elastic,
                                 rigid_body_sets, num_rigids, is_elastic_element, is_boundary_vertex, is_rigid_vertex,
                                 vertex_rigid_body);
  });
}
int mlx_wait_probe(int32_t device, int32_t kind, int64_t limit_ns, int32_t* timed_out) {
  return mlx::guarded([&]() -> int {
    if (!timed_out) return set_error(MLX_ERR_ARGUMENT, "null argument");
    if (kind != 0 && kind != 1) return set_error(MLX_ERR_ARGUMENT, "kind must be 0 (grid barrier) or 1 (mbarrier)");
    limit_ns = std::max<int64_t>(1000000, std::min<int64_t>(limit_ns, 2000000000));
    *timed_out = 0;
    if (kind == 1) return mlx::mlp_wait_probe(device, (long long)limit_ns, timed_out);
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return set_error(MLX_ERR_ARGUMENT, "bad device");
    unsigned* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(unsigned) * 4);
    if (e == cudaSuccess) {
      cudaMemset(d, 0, sizeof(unsigned) * 4);
      k_probe_grid_wait<<<1, 32>>>(d, reinterpret_cast<int*>(d + 1), (unsigned long long)limit_ns,
                                   reinterpret_cast<int*>(d + 2));
      e = cudaGetLastError();
      int r = 0;
      if (e == cudaSuccess) e = cudaMemcpy(&r, d + 2, sizeof(int), cudaMemcpyDeviceToHost);
      *timed_out = r;
      cudaFree(d);
    }
    cudaSetDevice(prev);
    if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("grid wait probe: ") + cudaGetErrorString(e));
    return MLX_OK;
  });
}
int mlx_pcg_solve(mlx_solver* s, double h, const double* b, int32_t iterations, double* x, double* resvec) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->pcg_solve(h, b, iterations, x, resvec);
  });
}
int mlx_sim_contact_count(mlx_solver* s, int32_t* n) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver");
    return s->impl->sim_contact_count(n);
  });
}
int mlx_launch_path(const mlx_solver* s, char* buf, int32_t n) {
  return mlx::guarded([&]() -> int {
    if (!s) return set_error(MLX_ERR_ARGUMENT, "null solver"), -1;
    std::string d = s->impl->launch_path();
    if (buf && n > 0) {
      size_t k = std::min<size_t>(d.size(), (size_t)n - 1);
      std::memcpy(buf, d.data(), k);
      buf[k] = 0;
    }
    return (int)d.size();
  });
}

}  // extern "C"
