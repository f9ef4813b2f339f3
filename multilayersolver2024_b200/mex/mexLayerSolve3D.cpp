// mexLayerSolve3D.cpp -- MATLAB gateway of the B200 layer solve.
//
//   [xi, sumNonMonitoredTime, residualArray, runUntilResSmallerThan] = ...
//       mexLayerSolve3D(<the 50 arguments of xpbdLayer3D.layerSolve>)
//
// Same argument order, types and results as the static
// xpbdLayer3D.layerSolve (3d/integrator/xpbdLayer3D.m:44-93), so
// xpbdLayer3D.integrate (xpbdLayer3D.m:684) swaps one call.  The gateway keeps
// one device-resident solver per mesh (re-created when the mesh arrays
// change) and converts MATLAB doubles to the int32 ids of the C ABI.
// Precision: FP32 bulk projection unless the environment variable
// MLXPBD_PRECISION is "fp64".
//
// Build with MATLAB:  mex -R2018a mexLayerSolve3D.cpp -I<repo>/include
//                      -L<repo>/multilayersolver2024_b200 -lmlxpbd
#include "mex.h"
#include "mlxpbd.h"

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct MeshKey {
  const void* ptrs[9] = {nullptr};
  size_t N = 0, T = 0;
  int precision = 0;
  bool operator==(const MeshKey& o) const {
    return std::memcmp(ptrs, o.ptrs, sizeof(ptrs)) == 0 && N == o.N && T == o.T && precision == o.precision;
  }
};

mlx_solver* g_solver = nullptr;
MeshKey g_key;

void release() {
  if (g_solver) mlx_destroy(g_solver);
  g_solver = nullptr;
}

[[noreturn]] void fail(const char* id, const std::string& msg) {
  mexErrMsgIdAndTxt(id, "%s", msg.c_str());
  std::abort();  // not reached: mexErrMsgIdAndTxt does not return
}

double scalar(const mxArray* a) { return mxGetScalar(a); }

std::vector<int32_t> to_i32(const mxArray* a) {
  size_t n = mxGetNumberOfElements(a);
  std::vector<int32_t> v(n);
  if (mxIsInt32(a)) {
    std::memcpy(v.data(), mxGetInt32s(a), n * sizeof(int32_t));
  } else if (mxIsDouble(a)) {
    const double* d = mxGetDoubles(a);
    for (size_t i = 0; i < n; ++i) v[i] = (int32_t)d[i];
  } else if (mxIsLogical(a)) {
    const mxLogical* l = mxGetLogicals(a);
    for (size_t i = 0; i < n; ++i) v[i] = l[i] ? 1 : 0;
  } else {
    fail("MLXPBD:type", "expected a double, int32 or logical array");
  }
  return v;
}

std::vector<uint8_t> to_u8(const mxArray* a) {
  size_t n = mxGetNumberOfElements(a);
  std::vector<uint8_t> v(n);
  if (mxIsLogical(a)) {
    const mxLogical* l = mxGetLogicals(a);
    for (size_t i = 0; i < n; ++i) v[i] = l[i] ? 1 : 0;
  } else if (mxIsDouble(a)) {
    const double* d = mxGetDoubles(a);
    for (size_t i = 0; i < n; ++i) v[i] = d[i] != 0;
  } else {
    fail("MLXPBD:type", "expected a logical mask");
  }
  return v;
}

const double* dbl(const mxArray* a, size_t n, const char* what) {
  if (!mxIsDouble(a) || mxIsComplex(a)) fail("MLXPBD:type", std::string(what) + " must be real double");
  if (mxGetNumberOfElements(a) < n) fail("MLXPBD:size", std::string(what) + " is too small");
  return mxGetDoubles(a);
}

}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 50) mexErrMsgIdAndTxt("MLXPBD:nrhs", "50 inputs required (the arguments of xpbdLayer3D.layerSolve).");
  if (nlhs > 4) mexErrMsgIdAndTxt("MLXPBD:nlhs", "at most 4 outputs.");
  // 1-based positions of the reference's argument list
  const mxArray* a[51];
  for (int i = 0; i < 50; ++i) a[i + 1] = prhs[i];
  const mxArray* tArr = a[31];
  if (!mxIsInt32(tArr) || mxGetN(tArr) != 4) fail("MLXPBD:T", "T must be an int32 T x 4 array");
  const size_t T = mxGetM(tArr);
  const size_t N = mxGetNumberOfElements(a[7]) / 3;
  const size_t L = mxGetNumberOfElements(a[17]);          // layers
  const size_t Ls = T ? mxGetNumberOfElements(a[3]) / T : 0;  // sorted layer columns
  const size_t Lv = N ? mxGetNumberOfElements(a[4]) / N : 0;  // columns of the vertex masks
  const size_t K = mxGetNumberOfElements(a[29]);
  if (L == 0 || Ls == 0 || Lv < Ls) fail("MLXPBD:layers", "layer arrays are inconsistent");

  const char* prec = std::getenv("MLXPBD_PRECISION");
  const int precision = (prec && std::string(prec) == "fp64") ? MLX_FP64 : MLX_FP32;

  // ---- mesh (cached across calls while the arrays stay the same) ----
  std::vector<int32_t> color = to_i32(a[37]);
  std::vector<int32_t> pinned = to_i32(a[33]);
  MeshKey key;
  const mxArray* meshArgs[9] = {a[30], a[31], a[34], a[35], a[45], a[46], a[37], a[33], a[39]};
  for (int i = 0; i < 9; ++i) key.ptrs[i] = mxGetData(meshArgs[i]);
  key.N = N;
  key.T = T;
  key.precision = precision;
  if (!g_solver || !(key == g_key)) {
    release();
    mlx_mesh_desc md;
    std::memset(&md, 0, sizeof(md));
    md.num_vertices = (int32_t)N;
    md.num_tets = (int32_t)T;
    md.t = mxGetInt32s(tArr);
    md.mass = dbl(a[30], 3 * N, "mass");
    md.DmInv = dbl(a[34], 9 * T, "DmInv");
    md.volume = dbl(a[46], T, "volume");
    md.element_color = color.data();
    md.num_colors = (int32_t)scalar(a[39]);
    md.pinned_dofs = pinned.data();
    md.num_pinned_dofs = (int32_t)pinned.size();
    md.energy_type = MLX_ENERGY_STVK_VOIGT;  // the reference's 3D constraint
    md.alpha = dbl(a[35], 36 * T, "perElementXPBDalphaMatrix");
    md.beta = dbl(a[45], 36 * T, "perElementXPBDBeta");
    md.precision = precision;
    md.device = 0;
    if (mlx_create(&md, &g_solver) != MLX_OK) {
      g_solver = nullptr;
      fail("MLXPBD:create", mlx_last_error());
    }
    g_key = key;
    mexAtExit(release);
  }

  // ---- per-call layer description ----
  std::vector<uint8_t> isE = to_u8(a[1]), isR = to_u8(a[2]), isBV = to_u8(a[5]), isRV = to_u8(a[6]);
  std::vector<int32_t> sets = to_i32(a[3]), vrb = to_i32(a[4]), numRigids = to_i32(a[11]);
  std::vector<int32_t> iterations = to_i32(a[16]), layersMap = to_i32(a[41]);
  mlx_layer_desc ld;
  ld.num_layers = (int32_t)L;
  ld.num_columns = (int32_t)Ls;
  ld.layers_map = layersMap.data();
  ld.iterations = iterations.data();
  ld.is_elastic_element = isE.data();
  ld.is_rigid_element = isR.data();
  ld.rigid_body_sets = sets.data();
  ld.vertex_rigid_body = vrb.data();
  ld.is_boundary_vertex = isBV.data();
  ld.is_rigid_vertex = isRV.data();
  ld.num_rigids = numRigids.data();

  mlx_solve_params P = {};  // contact_coloring 0: the reference's order
  P.h = scalar(a[10]);
  P.boundary_compliance = scalar(a[13]);
  P.contact_resistance = scalar(a[14]);
  P.run_until = scalar(a[18]);
  P.give_up_threshold = scalar(a[22]);
  P.gravity_compliance = scalar(a[42]);
  P.gravity = scalar(a[43]);
  P.stop_at_improvement_percent = scalar(a[49]);
  P.compute_residuals = scalar(a[19]) != 0;
  P.hanging_stop = (int32_t)scalar(a[20]);
  P.give_up_enabled = scalar(a[21]) != 0;
  P.last_layer_give_up_enabled = scalar(a[23]) != 0;
  P.use_gravity_constraints = scalar(a[24]) != 0;
  P.use_rigid_contacts = scalar(a[48]) != 0;

  std::vector<int32_t> cvid = to_i32(a[29]);
  mlx_contacts C;
  C.num_contacts = (int32_t)K;
  C.normals = K ? dbl(a[27], 3 * K, "contactNormals") : nullptr;
  C.point_colliders = K ? dbl(a[28], 3 * K, "pointColliders") : nullptr;
  C.vertex_ids = cvid.data();
  C.compliance = K ? dbl(a[15], K, "contactCompliance") : nullptr;

  const size_t nres = mxGetNumberOfElements(a[12]);
  mlx_solve_inputs in;
  in.xi = dbl(a[7], 3 * N, "xi");
  in.lambdai = dbl(a[8], 6 * T, "lambdai");
  in.oldp = dbl(a[25], 3 * N, "oldp");
  in.old_oldp = dbl(a[26], 3 * N, "oldOldp");
  in.f = dbl(a[40], 3 * N, "f");
  in.residualv = dbl(a[44], 3 * N, "residualv");
  in.pinnedx = pinned.empty() ? nullptr : dbl(a[50], pinned.size(), "pinnedx");
  in.residual_in = nres ? dbl(a[12], nres, "residualArray") : nullptr;
  in.residual_in_len = (int32_t)nres;
  in.sum_non_monitored_time = scalar(a[9]);

  // residualArray can grow by one entry per iteration
  long long cap = (long long)nres + 1;
  for (size_t l = 0; l < L; ++l) cap += iterations[l];
  if (P.hanging_stop >= 0) cap += P.hanging_stop;
  if (P.run_until >= 0 && P.hanging_stop < 0) cap += 1000000;
  std::vector<double> residual((size_t)cap);
  plhs[0] = mxCreateDoubleMatrix(3 * N, 1, mxREAL);
  mlx_solve_outputs out;
  std::memset(&out, 0, sizeof(out));
  out.xi = mxGetDoubles(plhs[0]);
  out.lambdai = nullptr;
  out.residual = residual.data();
  out.residual_capacity = (int32_t)cap;
  if (mlx_layer_solve(g_solver, &ld, &P, &C, &in, &out) != MLX_OK) fail("MLXPBD:solve", mlx_last_error());
  if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(out.sum_non_monitored_time);
  if (nlhs > 2) {
    plhs[2] = mxCreateDoubleMatrix(1, out.residual_len, mxREAL);
    if (out.residual_len) std::memcpy(mxGetDoubles(plhs[2]), residual.data(), sizeof(double) * out.residual_len);
  }
  if (nlhs > 3) plhs[3] = mxCreateDoubleScalar(out.run_until);
}
