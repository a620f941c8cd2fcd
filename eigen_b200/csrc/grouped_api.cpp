// grouped_api.cpp -- eb2_grouped_plan_* / eb2_gemm_grouped: validation, descriptor
// upload, the tile schedule (longest K first) and CUDA-graph capture of the launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "context.h"
#include "eigen_b200/blas.h"
#include "grouped.h"
#include "kernels.h"
#include "mlp.h"

struct eb2_grouped_plan {
  int device = -1;
  bool f64 = true;
  int64_t count = 0, num_items = 0;
  eb2::GroupedProblem* d_problems = nullptr;
  eb2::GroupedItem* d_items = nullptr;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool classes_on = true;  // products share warps (size classes), else 32 x 32 tiles only
};

namespace eb2 {
namespace {

int op_code(char c) {
  if (c == 'N' || c == 'n') return 0;
  if (c == 'T' || c == 't' || c == 'C' || c == 'c') return 1;
  return -1;
}

void release(eb2_grouped_plan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  if (p->d_problems) cudaFree(p->d_problems);
  if (p->d_items) cudaFree(p->d_items);
  delete p;
}

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  (void)cudaGetLastError();
  set_error(EB2_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

// The size classes of a plan: the caller's setting, else a forced configuration class (the
// tuner), else the learned picker on the batch's geometric-mean shape and count, else 8 / 16.
GroupedClasses resolve_classes(char dtype, int64_t count, const eb2_gemm_problem* ps) {
  GroupedClasses c = grouped_classes();
  if (!c.automatic) return c;
  c.small_max = 8;
  c.mid_max = 16;
  int cfg = forced_config();
  if (cfg != kCfgBatchClasses && cfg != kCfgBatchTiles) {
    cfg = -1;
    if (picker_weights() != nullptr && count > 1) {
      double lm = 0, ln = 0, lk = 0;
      int64_t used = 0;
      for (int64_t i = 0; i < count; ++i) {
        if (ps[i].m <= 0 || ps[i].n <= 0) continue;
        lm += std::log(double(ps[i].m));
        ln += std::log(double(ps[i].n));
        lk += std::log(double(std::max<int64_t>(ps[i].k, 1)));
        ++used;
      }
      int cls = 0;
      if (used > 0)
        (void)picker_predict(int64_t(std::llround(std::exp(lm / used))), int64_t(std::llround(std::exp(ln / used))),
                             int64_t(std::llround(std::exp(lk / used))), dtype, 0.0, count,
                             dtype == 'd' ? 1.1102230246251565e-16 : 5.9604644775390625e-08, &cfg, &cls);
    }
  }
  if (cfg == kCfgBatchTiles) c.small_max = c.mid_max = 0;
  return c;
}

// Validates and converts the problems; builds the work items in schedule order: products of
// at most small_max x small_max four to a warp, of at most mid_max two to a warp (each group
// of similar K), larger ones cut into 32 x 32 tiles; then all items longest-K first.
int build(char dtype, int64_t count, const eb2_gemm_problem* ps, std::vector<GroupedProblem>& out,
          std::vector<GroupedItem>& items, bool* classes_on = nullptr) {
  out.resize(size_t(count));
  std::vector<std::pair<int64_t, GroupedItem>> keyed;
  std::vector<std::pair<int64_t, uint32_t>> small, mid;  // (k, problem) of the shared-warp classes
  const GroupedClasses cls = resolve_classes(dtype, count, ps);
  if (classes_on) *classes_on = cls.small_max > 0 || cls.mid_max > 0;
  for (int64_t i = 0; i < count; ++i) {
    const eb2_gemm_problem& q = ps[i];
    const int oa = op_code(q.transa), ob = op_code(q.transb);
    // the BLAS argument rules of blas/level3_impl.h:61-78
    int info = 0;
    if (oa < 0) info = 1;
    else if (ob < 0) info = 2;
    else if (q.m < 0) info = 3;
    else if (q.n < 0) info = 4;
    else if (q.k < 0) info = 5;
    else if (q.lda < std::max<int64_t>(1, oa == 0 ? q.m : q.k)) info = 8;
    else if (q.ldb < std::max<int64_t>(1, ob == 0 ? q.k : q.n)) info = 10;
    else if (q.ldc < std::max<int64_t>(1, q.m)) info = 13;
    if (info) {
      set_error(EB2_ERR_ARG, "grouped %cGEMM problem %lld: invalid argument (BLAS info %d)", dtype == 'd' ? 'D' : 'S',
                static_cast<long long>(i), info);
      return EB2_ERR_ARG;
    }
    if ((q.m + 31) / 32 > 65535 || (q.n + 31) / 32 > 65535) {
      set_error(EB2_ERR_ARG, "grouped problem %lld is too large for the batched path", static_cast<long long>(i));
      return EB2_ERR_ARG;
    }
    GroupedProblem& g = out[size_t(i)];
    g.m = q.m;
    g.n = q.n;
    g.k = (q.alpha == 0.0) ? 0 : q.k;  // alpha == 0: A and B are not read
    g.lda = q.lda;
    g.ldb = q.ldb;
    g.ldc = q.ldc;
    g.a = q.a;
    g.b = q.b;
    g.c = q.c;
    g.alpha = q.alpha;
    g.beta = q.beta;
    g.trans = (oa ? 1 : 0) | (ob ? 2 : 0);
    g.pad_ = 0;
    if (q.m == 0 || q.n == 0) continue;
    if (g.k == 0 && q.beta == 1.0) continue;  // nothing to do
    const int64_t side = std::max(q.m, q.n);
    if (side <= cls.small_max) {
      small.push_back({g.k, uint32_t(i)});
    } else if (side <= cls.mid_max) {
      mid.push_back({g.k, uint32_t(i)});
    } else {
      const int tm = int((q.m + 31) / 32), tn = int((q.n + 31) / 32);
      for (int a = 0; a < tn; ++a)
        for (int b = 0; b < tm; ++b) {
          GroupedItem it{};
          it.problem[0] = uint32_t(i);
          it.problem[1] = it.problem[2] = it.problem[3] = kNoProblem;
          it.k = int32_t(std::min<int64_t>(g.k, INT32_MAX));
          it.tile_m = uint16_t(b);
          it.tile_n = uint16_t(a);
          it.cls = 32;
          keyed.push_back({g.k, it});
        }
    }
  }
  // products that share a warp: similar K together (each item walks its largest K)
  auto pack = [&](std::vector<std::pair<int64_t, uint32_t>>& v, int per_item, uint8_t c) {
    std::stable_sort(v.begin(), v.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    for (size_t s = 0; s < v.size(); s += size_t(per_item)) {
      GroupedItem it{};
      for (int q = 0; q < 4; ++q) it.problem[q] = kNoProblem;
      for (int q = 0; q < per_item && s + size_t(q) < v.size(); ++q) it.problem[q] = v[s + size_t(q)].second;
      it.k = int32_t(std::min<int64_t>(v[s].first, INT32_MAX));
      it.cls = c;
      keyed.push_back({v[s].first, it});
    }
  };
  pack(small, 4, 8);
  pack(mid, 2, 16);
  // longest K first: a greedy balance of the uneven work over the persistent warps
  std::stable_sort(keyed.begin(), keyed.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  items.resize(keyed.size());
  for (size_t i = 0; i < keyed.size(); ++i) items[i] = keyed[i].second;
  return EB2_OK;
}

}  // namespace

GroupedClasses& grouped_classes() {
  static GroupedClasses c;
  return c;
}

}  // namespace eb2

extern "C" {

int eb2_grouped_plan_create(char dtype, int64_t count, const eb2_gemm_problem* problems, eb2_grouped_plan_t* plan) {
  if (!plan || count < 0 || (count > 0 && !problems) || (dtype != 'd' && dtype != 's')) {
    eb2::set_error(EB2_ERR_ARG, "eb2_grouped_plan_create: invalid arguments");
    return EB2_ERR_ARG;
  }
  *plan = nullptr;
  eb2::Context* cx = eb2::current_context();
  if (!cx) return EB2_ERR_NO_DEVICE;
  std::vector<eb2::GroupedProblem> ps;
  std::vector<eb2::GroupedItem> items;
  bool classes_on = true;
  int rc = eb2::build(dtype, count, problems, ps, items, &classes_on);
  if (rc != EB2_OK) return rc;
  auto* p = new eb2_grouped_plan();
  p->classes_on = classes_on;
  p->device = cx->device;
  p->f64 = (dtype == 'd');
  p->count = count;
  p->num_items = int64_t(items.size());
  bool ok = eb2::cuda_ok(cudaMalloc(&p->d_problems, std::max<size_t>(1, ps.size()) * sizeof(eb2::GroupedProblem)),
                         "grouped descriptors");
  ok = ok && eb2::cuda_ok(cudaMalloc(&p->d_items, std::max<size_t>(1, items.size()) * sizeof(eb2::GroupedItem)),
                          "grouped schedule");
  ok = ok && eb2::cuda_ok(cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking), "capture stream");
  if (ok && !ps.empty())
    ok = eb2::cuda_ok(cudaMemcpy(p->d_problems, ps.data(), ps.size() * sizeof(eb2::GroupedProblem),
                                 cudaMemcpyHostToDevice),
                      "upload descriptors");
  if (ok && !items.empty())
    ok = eb2::cuda_ok(cudaMemcpy(p->d_items, items.data(), items.size() * sizeof(eb2::GroupedItem),
                                 cudaMemcpyHostToDevice),
                      "upload schedule");
  unsigned blocks = 0;
  ok = ok && eb2::cuda_ok(eb2::grouped_grid(p->f64, p->num_items, cx->num_sms, &blocks), "grouped grid");
  if (ok) {
    ok = eb2::cuda_ok(cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    if (ok) {
      cudaError_t le = eb2::launch_grouped_gemm(p->f64, p->d_problems, p->d_items, p->num_items, blocks,
                                               p->capture_stream);
      cudaError_t ee = cudaStreamEndCapture(p->capture_stream, &p->graph);
      ok = eb2::cuda_ok(le, "grouped launch (capture)") && eb2::cuda_ok(ee, "end capture");
    }
    ok = ok && eb2::cuda_ok(cudaGraphInstantiate(&p->exec, p->graph, 0), "instantiate graph");
  }
  if (!ok) {
    eb2::release(p);
    return EB2_ERR_CUDA;
  }
  *plan = p;
  return EB2_OK;
}

int eb2_grouped_plan_execute(eb2_grouped_plan_t plan, void* stream) {
  if (!plan) {
    eb2::set_error(EB2_ERR_ARG, "eb2_grouped_plan_execute: null plan");
    return EB2_ERR_ARG;
  }
  eb2_call_info& ci = eb2::call_info();
  ci = eb2_call_info{};
  eb2::call_config() = eb2::CallConfig{};
  eb2::call_config().config = plan->classes_on ? eb2::kCfgBatchClasses : eb2::kCfgBatchTiles;
  ci.dtype = plan->f64 ? 'd' : 's';
  ci.method = EB2_METHOD_NATIVE;
  ci.launches = plan->num_items > 0 ? 1 : 0;
  ci.err_estimate = -1.0;
  ci.kernel_ms = -1.0;
  ci.gemm_kernel_ms = -1.0;
  if (plan->num_items == 0) return EB2_OK;
  return eb2::cuda_ok(cudaGraphLaunch(plan->exec, static_cast<cudaStream_t>(stream)), "grouped graph launch")
             ? EB2_OK
             : EB2_ERR_CUDA;
}

int eb2_grouped_plan_destroy(eb2_grouped_plan_t plan) {
  if (plan) cudaDeviceSynchronize();
  eb2::release(plan);
  return EB2_OK;
}

int eb2_gemm_grouped(char dtype, int64_t count, const eb2_gemm_problem* problems, void* stream) {
  eb2_grouped_plan_t plan = nullptr;
  int rc = eb2_grouped_plan_create(dtype, count, problems, &plan);
  if (rc != EB2_OK) return rc;
  rc = eb2_grouped_plan_execute(plan, stream);
  if (rc == EB2_OK && !eb2::cuda_ok(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "grouped GEMM"))
    rc = EB2_ERR_CUDA;
  eb2_grouped_plan_destroy(plan);
  return rc;
}

int eb2_gemm_each(char dtype, int64_t count, const eb2_gemm_problem* problems, void* stream) {
  if (count < 0 || (count > 0 && !problems) || (dtype != 'd' && dtype != 's')) {
    eb2::set_error(EB2_ERR_ARG, "eb2_gemm_each: invalid arguments");
    return EB2_ERR_ARG;
  }
  std::vector<eb2::GroupedProblem> ps;
  std::vector<eb2::GroupedItem> items;
  int rc = eb2::build(dtype, count, problems, ps, items);  // same validation as the grouped path
  if (rc != EB2_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int64_t i = 0; i < count; ++i) {
    const eb2_gemm_problem& q = problems[i];
    if (q.m == 0 || q.n == 0) continue;
    const bool ta = eb2::op_code(q.transa) != 0, tb = eb2::op_code(q.transb) != 0;
    cudaError_t e;
    if (dtype == 'd') {
      // the FP64 kernel of the grouped launch walks K in the native kernel's order: the plain
      // native DGEMM gives the same bits
      if (q.k == 0 || q.alpha == 0.0)
        e = q.beta == 1.0 ? cudaSuccess : eb2::launch_scale_matrix_d(q.m, q.n, q.beta, static_cast<double*>(q.c), q.ldc, st);
      else
        e = eb2::launch_dgemm_native(ta, tb, q.m, q.n, q.k, q.alpha, static_cast<const double*>(q.a), q.lda,
                                     static_cast<const double*>(q.b), q.ldb, q.beta, static_cast<double*>(q.c), q.ldc,
                                     nullptr, st);
    } else {
      // FP32: the split-BF16 tile arithmetic of the grouped launch, one launch per product
      const eb2::GroupedProblem& g = ps[size_t(i)];
      e = (g.k == 0 && g.beta == 1.0) ? cudaSuccess : eb2::launch_grouped_one(false, g, st);
    }
    if (!eb2::cuda_ok(e, "per-product launch")) return EB2_ERR_CUDA;
  }
  return EB2_OK;
}

int eb2_set_grouped_classes(int small_max, int mid_max) {
  if (small_max == -1 && mid_max == -1) {
    eb2::grouped_classes() = eb2::GroupedClasses{};
    return EB2_OK;
  }
  if (small_max < 0 || small_max > 8 || mid_max < 0 || mid_max > 16) {
    eb2::set_error(EB2_ERR_ARG, "eb2_set_grouped_classes: small_max in [0, 8], mid_max in [0, 16] (or both -1)");
    return EB2_ERR_ARG;
  }
  eb2::grouped_classes().small_max = small_max;
  eb2::grouped_classes().mid_max = mid_max;
  eb2::grouped_classes().automatic = false;
  return EB2_OK;
}

}  // extern "C"
