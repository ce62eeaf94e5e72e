// hbx_api.cu -- the hbx_* C API and the HACApK drop-in entry points.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/hacapk_b200.h"
#include "hbx_engine.h"
#include "hbx_flat.h"

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string &msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? HBX_ERR_NOMEM : HBX_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

// Every device allocation of the library goes through dev_malloc.  A test
// hook (hbx_debug_fail_alloc) can make the n-th one from now fail as
// cudaMalloc does when the device is out of memory, so the error paths that
// release a half-built engine run without exhausting a real GPU.
std::atomic<int> g_fail_alloc{-1};
cudaError_t dev_malloc(void *p, size_t bytes) {
  int n = g_fail_alloc.load();
  while (n >= 0) {
    if (g_fail_alloc.compare_exchange_weak(n, n - 1)) {
      if (n == 0) return cudaErrorMemoryAllocation;
      break;
    }
  }
  return cudaMalloc(reinterpret_cast<void **>(p), bytes);
}

#define HBX_CUDA(call)                               \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void free_engine(hbx_hmat *h) {
  if (!h) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  cudaFree(h->d_stream);
  cudaFree(h->d_recs);
  cudaFree(h->d_ctas);
  cudaFree(h->d_lite);
  cudaFree(h->d_atoms);
  cudaFree(h->d_zbu);
  cudaFree(h->d_gbar);
  cudaFree(h->d_err);
  cudaFree(h->d_prof);
  cudaFree(h->d_x);
  cudaFree(h->d_y);
  cudaFree(h->d_work);
  cudaFree(h->d_part);
  cudaFree(h->d_dot);
  cudaFree(h->d_state);
  cudaFree(h->d_hist);
  cudaFree(h->d_refine);
  cudaFree(h->d_gcr);
  cudaFree(h->d_chunk_inst);
  cudaFree(h->d_rflag);
  cudaFree(h->d_chunk_base);
  cudaFree(h->d_inst_pre);
  cudaFree(h->d_pipe);
  cudaFree(h->d_pstate);
  cudaFree(h->d_ppart);
  cudaFree(h->d_phist);
  if (h->h_pstate) cudaFreeHost(h->h_pstate);
  if (h->pgraph) cudaGraphExecDestroy(h->pgraph);
  cudaFree(h->d_gcrs);
  cudaFree(h->d_gcrpart);
  if (h->h_gcrs) cudaFreeHost(h->h_gcrs);
  if (h->ggraph) cudaGraphExecDestroy(h->ggraph);
  cudaFree(h->d_f32);
  cudaFree(h->d_zbum);
  cudaFree(h->d_mrv);
  cudaFree(h->d_mr32);
  cudaFree(h->d_mrpart);
  cudaFree(h->d_mrsc);
  cudaFree(h->d_mrint);
  cudaFree(h->d_mrdbl);
  if (h->h_mrpin) cudaFreeHost(h->h_mrpin);
  cudaFree(h->d_inst_off);
  cudaFree(h->d_rinst);
  cudaFree(h->d_btv);
  cudaFree(h->d_btsc);
  cudaFree(h->d_btdbl);
  cudaFree(h->d_btany);
  if (h->h_pin) cudaFreeHost(h->h_pin);
  if (h->h_state) cudaFreeHost(h->h_state);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->ev2) cudaEventDestroy(h->ev2);
  if (h->ev3) cudaEventDestroy(h->ev3);
  if (h->ev4) cudaEventDestroy(h->ev4);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (cur >= 0 && cur != h->device) cudaSetDevice(cur);
  delete h;
}

// Reads and clears the device error word; resets the grid barrier after a
// failure so the next launch starts from a clean state.
int check_device_error(hbx_hmat *h, cudaStream_t s) {
  int err = 0;
  cudaError_t e = cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "device error readback");
  if (err != 0) {
    cudaMemsetAsync(h->d_err, 0, sizeof(int), s);
    cudaMemsetAsync(h->d_gbar, 0, 2 * sizeof(unsigned), s);
    cudaStreamSynchronize(s);
    return fail(HBX_ERR_TIMEOUT, "a bounded device wait expired (error bits " + std::to_string(err) + ")");
  }
  return HBX_OK;
}

hbx::MatvecArgs matvec_args(hbx_hmat *h, double alpha, const double *x, double beta, const double *yin, double *y) {
  hbx::MatvecArgs a{};
  a.stream = h->d_stream;
  a.recs = h->d_recs;
  a.ctas = h->d_ctas;
  a.lite = h->d_lite;
  a.x = x;
  a.yin = yin;
  a.y = y;
  a.zbu = h->d_zbu;
  a.zbu_len = h->plan.zbu_len;
  if (h->d_f32) {
    a.x32 = h->d_f32;
    a.zbu32 = h->d_f32 + 3 * (size_t)h->plan.nd;
  }
  a.alpha = alpha;
  a.beta = beta;
  a.gbar = h->d_gbar;
  a.err = h->d_err;
  a.timeout_ns = h->timeout_ns;
  a.prof = h->d_prof;
  a.keep_frac = h->keep_frac;
  a.stall = h->stall_next;  // test hook: one launch only
  h->stall_next = 0;
  if (h->skip_inactive && h->d_chunk_inst) {
    a.chunk_inst = h->d_chunk_inst;
    a.chunk_base = h->d_chunk_base;
    a.inst_pre = h->d_inst_pre;
  }
  return a;
}

// One H-matvec launch; an FP32 or BF16 engine first rounds x into its float copy.
cudaError_t mv_launch(hbx_hmat *h, const hbx::MatvecArgs &a, cudaStream_t s) {
  if (h->plan.precision != hbx::kFP64) {
    cudaError_t e = hbx::launch_to_float(a.x, h->d_f32, (size_t)h->plan.nd, s);
    if (e != cudaSuccess) return e;
  }
  return hbx::launch_matvec(a, h->num_ctas, s, h->plan.precision);
}

int ensure_host_staging(hbx_hmat *h) {
  const size_t n = (size_t)h->plan.nd;
  if (!h->d_x) HBX_CUDA(dev_malloc(&h->d_x, n * sizeof(double)));
  if (!h->d_y) HBX_CUDA(dev_malloc(&h->d_y, n * sizeof(double)));
  if (!h->h_pin) HBX_CUDA(cudaHostAlloc(&h->h_pin, 2 * n * sizeof(double), cudaHostAllocDefault));
  return HBX_OK;
}

int ensure_solver(hbx_hmat *h, int max_iter) {
  const size_t n = (size_t)h->plan.nd;
  if (!h->d_work) HBX_CUDA(dev_malloc(&h->d_work, 8 * n * sizeof(double)));
  if (!h->d_part) HBX_CUDA(dev_malloc(&h->d_part, (size_t)h->num_ctas * hbx::kSlots * 2 * sizeof(double)));
  if (!h->d_dot) HBX_CUDA(dev_malloc(&h->d_dot, 4 * sizeof(double)));
  if (!h->d_state) HBX_CUDA(dev_malloc(&h->d_state, sizeof(hbx::BicgState)));
  if (!h->h_state) HBX_CUDA(cudaHostAlloc(&h->h_state, sizeof(hbx::BicgState), cudaHostAllocDefault));
  if (h->hist_cap < max_iter + 1) {
    cudaFree(h->d_hist);
    h->d_hist = nullptr;
    HBX_CUDA(dev_malloc(&h->d_hist, (size_t)(max_iter + 1) * sizeof(double)));
    h->hist_cap = max_iter + 1;
  }
  return HBX_OK;
}

std::mutex g_table_mu;
std::unordered_map<const void *, hbx_hmat *> g_table;

}  // namespace

extern "C" {

const char *hbx_status_string(int status) {
  switch (status) {
    case HBX_OK: return "HBX_OK";
    case HBX_ERR_INVALID: return "HBX_ERR_INVALID";
    case HBX_ERR_NOMEM: return "HBX_ERR_NOMEM";
    case HBX_ERR_CUDA: return "HBX_ERR_CUDA";
    case HBX_ERR_TIMEOUT: return "HBX_ERR_TIMEOUT";
    case HBX_ERR_BREAKDOWN: return "HBX_ERR_BREAKDOWN";
    case HBX_ERR_NOT_CONVERGED: return "HBX_ERR_NOT_CONVERGED";
    case HBX_ERR_NONFINITE: return "HBX_ERR_NONFINITE";
    case HBX_ERR_UNSUPPORTED: return "HBX_ERR_UNSUPPORTED";
    default: return "HBX_ERR_UNKNOWN";
  }
}

const char *hbx_last_error(void) { return g_last_error.c_str(); }

static int create_engine(const stc_HACApK_leafmtxp *st, int nd, const hbx_options *opt, hbx_hmat **out,
                         bool keep_host_tables = false);
static void release_host_tables(hbx::Plan &P);

int hbx_create(const stc_HACApK_leafmtxp *st, int nd, const hbx_options *opt, hbx_hmat **out) {
  return create_engine(st, nd, opt, out);
}

int hbx_create_batch(const stc_HACApK_leafmtxp *const *st, const int *nd, int count, const hbx_options *opt,
                     hbx_hmat **out) {
  if (!out) return fail(HBX_ERR_INVALID, "hbx_create_batch: out is NULL");
  *out = nullptr;
  if (opt && opt->nrhs > 1) return fail(HBX_ERR_UNSUPPORTED, "hbx_create_batch: a batch engine takes one vector");
  hbx::CombinedLeaves cl;
  std::string err;
  int rc = hbx::combine_leaves(st, nd, count, cl, err);
  if (rc != HBX_OK) return fail(rc, "hbx_create_batch: " + err);
  hbx_hmat *h = nullptr;
  rc = create_engine(&cl.container, cl.off[count], opt, &h, true);
  if (rc != HBX_OK) return rc;
  h->inst_off = cl.off;
  std::vector<int> rinst((size_t)cl.off[count]);
  for (int k = 0; k < count; ++k)
    for (int i = cl.off[k]; i < cl.off[k + 1]; ++i) rinst[i] = k;
  cudaError_t e;
  if ((e = dev_malloc(&h->d_inst_off, (count + 1) * sizeof(int))) != cudaSuccess ||
      (e = dev_malloc(&h->d_rinst, rinst.size() * sizeof(int))) != cudaSuccess ||
      (e = cudaMemcpy(h->d_inst_off, cl.off.data(), (count + 1) * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(h->d_rinst, rinst.data(), rinst.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) {
    free_engine(h);
    return cuda_fail(e, "hbx_create_batch: instance tables");
  }
  std::vector<uint32_t> cinst, cbase;
  const bool table = count < 0xffff && hbx::chunk_instances(h->plan, rinst, cinst, cbase);
  release_host_tables(h->plan);
  if (table) {
    if ((e = dev_malloc(&h->d_chunk_inst, cinst.size() * sizeof(uint32_t))) != cudaSuccess ||
        (e = dev_malloc(&h->d_chunk_base, cbase.size() * sizeof(uint32_t))) != cudaSuccess ||
        (e = dev_malloc(&h->d_inst_pre, (count + 1) * sizeof(int))) != cudaSuccess ||
        (e = cudaMemcpy(h->d_chunk_inst, cinst.data(), cinst.size() * sizeof(uint32_t), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(h->d_chunk_base, cbase.data(), cbase.size() * sizeof(uint32_t), cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
      free_engine(h);
      return cuda_fail(e, "hbx_create_batch: chunk table");
    }
  }
  *out = h;
  return HBX_OK;
}

static void release_host_tables(hbx::Plan &P) {
  P.recs.clear();
  P.recs.shrink_to_fit();
  P.lite.clear();
  P.lite.shrink_to_fit();
  P.blocks.clear();
  P.blocks.shrink_to_fit();
  P.pieces.clear();
  P.pieces.shrink_to_fit();
}

// keep_host_tables: the host copies of the run records stay (the caller
// reads them, then calls release_host_tables).
static int create_engine(const stc_HACApK_leafmtxp *st, int nd, const hbx_options *opt, hbx_hmat **out,
                         bool keep_host_tables) {
  if (!out) return fail(HBX_ERR_INVALID, "hbx_create: out is NULL");
  *out = nullptr;
  if (!st) return fail(HBX_ERR_INVALID, "hbx_create: container is NULL");
  if (nd <= 0) return fail(HBX_ERR_INVALID, "hbx_create: nd <= 0");
  if (opt && opt->precision != HBX_FP64 && opt->precision != HBX_FP32 && opt->precision != HBX_BF16)
    return fail(HBX_ERR_UNSUPPORTED, "hbx_create: precision must be HBX_FP64, HBX_FP32 or HBX_BF16");
  const int nrhs = (opt && opt->nrhs > 1) ? opt->nrhs : 1;
  if (nrhs != 1 && nrhs != hbx::kNrhs) return fail(HBX_ERR_UNSUPPORTED, "hbx_create: nrhs must be 0, 1 or HBX_NRHS");
  if (nrhs > 1 && opt->precision != HBX_FP32)
    return fail(HBX_ERR_UNSUPPORTED, "hbx_create: a multi-RHS engine needs precision HBX_FP32");
  const double t0 = now_s();
  hbx_hmat *h = new (std::nothrow) hbx_hmat();
  if (!h) return fail(HBX_ERR_NOMEM, "hbx_create: host allocation");
  auto bail = [&](int st_) { free_engine(h); return st_; };
  cudaError_t e;
  if ((e = cudaGetDevice(&h->device)) != cudaSuccess) return bail(cuda_fail(e, "cudaGetDevice"));
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, h->device)) != cudaSuccess) return bail(cuda_fail(e, "cudaGetDeviceProperties"));
  if (prop.major < 10) return bail(fail(HBX_ERR_UNSUPPORTED, "hbx_create: needs an sm_100 device"));
  if ((e = hbx::configure_kernels()) != cudaSuccess) return bail(cuda_fail(e, "configure_kernels"));
  if ((e = hbx::configure_matmat()) != cudaSuccess) return bail(cuda_fail(e, "configure_matmat"));
  h->nrhs = nrhs;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device);
  if (!coop) return bail(fail(HBX_ERR_UNSUPPORTED, "hbx_create: device lacks cooperative launch"));
  const int max_ctas = prop.multiProcessorCount;  // one CTA per SM (shared-memory bound)
  int nc = (opt && opt->num_ctas > 0) ? opt->num_ctas : max_ctas;
  if (nc > max_ctas) return bail(fail(HBX_ERR_INVALID, "hbx_create: num_ctas exceeds co-resident CTAs"));
  h->num_ctas = nc;
  // L2 budget for the factor stream's pass-to-pass residency (MB): 24 by
  // default, HBX_L2_KEEP_MB overrides it (0 turns the cache hints off), a
  // nonzero hbx_options::l2_keep_mb overrides both (-1: no hints)
  const char *keep = std::getenv("HBX_L2_KEEP_MB");
  double keep_mb = keep ? std::atof(keep) : 24.0;
  if (opt && opt->l2_keep_mb != 0) keep_mb = opt->l2_keep_mb > 0 ? (double)opt->l2_keep_mb : 0.0;
  const char *tmo = std::getenv("HBX_TIMEOUT_MS");
  if (tmo) h->timeout_ns = (unsigned long long)(std::atof(tmo) * 1e6);
  const char *prof = std::getenv("HBX_PROFILE");
  if (prof && std::atoi(prof) > 0) {
    if ((e = dev_malloc(&h->d_prof, (size_t)nc * 16 * sizeof(unsigned long long))) != cudaSuccess)
      return bail(cuda_fail(e, "cudaMalloc(prof)"));
    cudaMemset(h->d_prof, 0, (size_t)nc * 16 * sizeof(unsigned long long));
  }

  std::string err;
  hbx::TransposedLeaves tleaves;  // H^T (host memory until the stream is packed)
  if (opt && opt->transpose) {
    int rc = hbx::transpose_leaves(st, nd, tleaves, err);
    if (rc != HBX_OK) return bail(fail(rc, "hbx_create: " + err));
    st = &tleaves.container;
    h->transposed = 1;
  }
  hbx::PlanCosts costs;
  if (opt && opt->block_cost > 0) costs.block = (uint64_t)opt->block_cost;
  if (opt && opt->run_cost > 0) costs.run = (uint64_t)opt->run_cost;
  const int prec = !opt ? hbx::kFP64
                        : (opt->precision == HBX_BF16 ? hbx::kBF16 : (opt->precision == HBX_FP32 ? hbx::kFP32 : hbx::kFP64));
  // merged D+U blocks (single-vector engines): the atoms with low-rank rows
  // that each CTA keeps split -- its first ones, whose D runs cover the wait
  // for the zbu grid barrier -- 4 by default (C1 L5: H-matvec 50.0 -> 49.4
  // us, BiCGSTAB step 124.9 -> 123.0 us), HBX_MERGE_KEEP overrides; < 0:
  // none merged
  int merge_keep = 4;
  if (const char *mk = std::getenv("HBX_MERGE_KEEP")) merge_keep = std::atoi(mk);
  if (opt && opt->merge != 0) merge_keep = opt->merge > 0 ? opt->merge - 1 : -1;  // the caller's choice
  if (nrhs > 1) merge_keep = -1;
  h->merge_keep = merge_keep;
  h->l2_keep_mb = keep_mb > 0.0 ? (int)keep_mb : 0;
  int st_plan = hbx::make_plan(st, nd, nc, h->plan, err, prec, nrhs > 1, costs, merge_keep);
  if (st_plan != HBX_OK) return bail(fail(st_plan, "hbx_create: " + err));
  const hbx::Plan &P = h->plan;
  // L2 residency of the factor stream: the head of every CTA's stream, in
  // all keep_mb megabytes, is read with the evict_last policy so that it
  // stays in L2 from one product to the next; the rest streams with
  // evict_first (HBX_L2_KEEP_MB; 0 = plain copies)
  if (keep_mb > 0.0 && P.total_bytes > 0) {
    const double f = keep_mb * 1e6 / (double)P.total_bytes;
    h->keep_frac = f >= 1.0 ? 65536u : (uint32_t)(f * 65536.0);
  }

  std::vector<uint8_t> host;
  try {
    host.resize(P.total_bytes);
  } catch (...) {
    return bail(fail(HBX_ERR_NOMEM, "hbx_create: host staging buffer"));
  }
  hbx::pack_plan(st, P, host.data());

  if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(cuda_fail(e, "stream"));
  cudaEventCreate(&h->ev0);
  cudaEventCreate(&h->ev1);
  cudaEventCreate(&h->ev2);
  cudaEventCreate(&h->ev3);
  cudaEventCreate(&h->ev4);
  if ((e = dev_malloc(&h->d_stream, P.total_bytes)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(stream)"));
  if ((e = dev_malloc(&h->d_recs, std::max<size_t>(1, P.recs.size()) * sizeof(hbx::RunRec))) != cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(run records)"));
  if ((e = dev_malloc(&h->d_ctas, P.ctas.size() * sizeof(hbx::CtaInfo))) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(ctas)"));
  if ((e = dev_malloc(&h->d_lite, std::max<size_t>(1, P.lite.size()) * sizeof(hbx::RunLite))) != cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(lite)"));
  if ((e = dev_malloc(&h->d_atoms, std::max<size_t>(1, P.atoms.size()) * sizeof(hbx::Atom))) != cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(atoms)"));
  // zbu twice: the two H-matvecs of a BiCGSTAB step write separate copies
  if ((e = dev_malloc(&h->d_zbu, 2 * std::max<uint64_t>(1, P.zbu_len) * sizeof(double))) != cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(zbu)"));
  if (P.precision != hbx::kFP64 &&
      (e = dev_malloc(&h->d_f32, (3 * (size_t)nd + 2 * std::max<uint64_t>(1, P.zbu_len)) * sizeof(float))) !=
          cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(float copies)"));
  if (nrhs > 1 &&
      (e = dev_malloc(&h->d_zbum, std::max<uint64_t>(1, P.zbu_len) * hbx::kNrhs * sizeof(float))) != cudaSuccess)
    return bail(cuda_fail(e, "cudaMalloc(multi-RHS zbu)"));
  if ((e = dev_malloc(&h->d_gbar, 4 * sizeof(unsigned))) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(gbar)"));
  if ((e = dev_malloc(&h->d_err, sizeof(int))) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(err)"));
  if ((e = cudaMemcpy(h->d_stream, host.data(), P.total_bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
    return bail(cuda_fail(e, "upload stream"));
  if (!P.recs.empty() &&
      (e = cudaMemcpy(h->d_recs, P.recs.data(), P.recs.size() * sizeof(hbx::RunRec), cudaMemcpyHostToDevice)) != cudaSuccess)
    return bail(cuda_fail(e, "upload run records"));
  if ((e = cudaMemcpy(h->d_ctas, P.ctas.data(), P.ctas.size() * sizeof(hbx::CtaInfo), cudaMemcpyHostToDevice)) != cudaSuccess)
    return bail(cuda_fail(e, "upload ctas"));
  if (!P.lite.empty() &&
      (e = cudaMemcpy(h->d_lite, P.lite.data(), P.lite.size() * sizeof(hbx::RunLite), cudaMemcpyHostToDevice)) !=
          cudaSuccess)
    return bail(cuda_fail(e, "upload run summaries"));
  if (!P.atoms.empty() &&
      (e = cudaMemcpy(h->d_atoms, P.atoms.data(), P.atoms.size() * sizeof(hbx::Atom), cudaMemcpyHostToDevice)) != cudaSuccess)
    return bail(cuda_fail(e, "upload atoms"));
  cudaMemset(h->d_gbar, 0, 4 * sizeof(unsigned));
  cudaMemset(h->d_err, 0, sizeof(int));
  cudaMemset(h->d_zbu, 0, 2 * std::max<uint64_t>(1, P.zbu_len) * sizeof(double));
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(cuda_fail(e, "hbx_create sync"));
  // host copies of the records and the packing tables are no longer needed
  h->num_runs = (long long)P.recs.size();
  if (!keep_host_tables) release_host_tables(h->plan);
  h->setup_seconds = now_s() - t0;
  *out = h;
  return HBX_OK;
}

int hbx_debug_stall_next_barrier(hbx_hmat *h) {
  if (!h) return fail(HBX_ERR_INVALID, "hbx_debug_stall_next_barrier: NULL handle");
  h->stall_next = 1;
  return HBX_OK;
}

int hbx_debug_fail_alloc(int n) {
  g_fail_alloc.store(n < 0 ? -1 : n);
  return HBX_OK;
}

int hbx_destroy(hbx_hmat *h) {
  if (!h) return fail(HBX_ERR_INVALID, "hbx_destroy: NULL handle");
  free_engine(h);
  return HBX_OK;
}

// Diagnostics: copies the per-CTA phase stamps of the last k_matvec
// (HBX_PROFILE=1 at create time) into out[num_ctas*8]; returns the count.
int hbx_debug_phase_stamps(hbx_hmat *h, unsigned long long *out, int cap) {
  if (!h || !out || !h->d_prof || cap <= 0) return 0;
  const int n = std::min(cap, h->num_ctas * 16);
  cudaDeviceSynchronize();
  cudaMemcpy(out, h->d_prof, (size_t)n * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  return n;
}

int hbx_get_info(const hbx_hmat *h, hbx_info *info) {
  if (!h || !info) return fail(HBX_ERR_INVALID, "hbx_get_info: NULL argument");
  std::memset(info, 0, sizeof(*info));
  const hbx::Plan &P = h->plan;
  info->nd = P.nd;
  info->nlf = P.nlf;
  info->nlfkt = P.nlfkt;
  info->ktmax = P.ktmax;
  info->num_ctas = h->num_ctas;
  info->num_atoms = (int)P.atoms.size();
  info->num_runs = (int)h->num_runs;
  info->precision = P.precision == hbx::kBF16 ? HBX_BF16 : (P.precision == hbx::kFP32 ? HBX_FP32 : HBX_FP64);
  uint64_t sb = 0;
  for (const auto &c : P.ctas) sb += c.stream_bytes;
  info->stream_bytes = (long long)sb;
  info->alg_bytes = (long long)P.alg_bytes;
  info->alg_flops = (long long)P.alg_flops;
  info->zbu_len = (long long)P.zbu_len;
  info->dense_words = (long long)P.dense_words;
  info->lowrank_words = (long long)P.lowrank_words;
  info->setup_seconds = h->setup_seconds;
  info->transposed = h->transposed;
  info->nrhs = h->nrhs;
  info->instances = h->inst_off.empty() ? 1 : (int)h->inst_off.size() - 1;
  info->block_cost = (int)P.costs.block;
  info->run_cost = (int)P.costs.run;
  info->merge_keep = h->merge_keep;
  info->l2_keep_mb = h->l2_keep_mb;
  return HBX_OK;
}

int hbx_autotune(const stc_HACApK_leafmtxp *st, int nd, const hbx_options *base, int reps, hbx_options *best,
                 double *best_us, double *default_us) {
  if (!st || nd <= 0) return fail(HBX_ERR_INVALID, "hbx_autotune: null container or nd <= 0");
  if (reps <= 0) reps = 20;
  hbx_options b0{};
  if (base) b0 = *base;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool multi = b0.nrhs > 1;
  const int nrows = nd;
  // vectors for the timed products (contents do not change the time)
  const size_t nx = (size_t)nrows * (multi ? hbx::kNrhs : 1);
  void *x = nullptr;
  double *y = nullptr;
  HBX_CUDA(dev_malloc(&x, nx * sizeof(double)));
  if (dev_malloc(&y, nx * sizeof(double)) != cudaSuccess) {
    cudaFree(x);
    return fail(HBX_ERR_NOMEM, "hbx_autotune: vectors");
  }
  cudaMemset(x, 0, nx * sizeof(double));
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // Stage 1: the CTA schedule (cost model, CTA count).  Stage 2, for
  // single-vector engines, from the best schedule: the merged D+U layout
  // (atoms kept split per CTA), then the L2 budget of the stream.
  struct Cand { int block, run, ctas, merge, l2; };
  std::vector<Cand> cands;
  for (int bc : {0, 2048, 32768})
    for (int rc : {0, 1024, 16384}) cands.push_back({bc, rc, 0, 0, 0});
  cands.push_back({0, 0, std::max(1, sms - 4), 0, 0});
  double t_best = 1e30, t_def = -1.0;
  hbx_options o_best = b0;
  int rc_all = HBX_OK;
  const size_t n_stage1 = cands.size();
  for (size_t ci = 0; ci < cands.size(); ++ci) {
    if (ci == n_stage1 && !multi) {  // stage 2a: merged D+U runs around the best schedule
      for (int m : {-1, 1, 3, 9}) cands.push_back({o_best.block_cost, o_best.run_cost, o_best.num_ctas, m, 0});
    }
    if (ci == n_stage1 + 4 && !multi) {  // stage 2b: the L2 budget around the best so far
      for (int l2 : {-1, 12, 48}) cands.push_back({o_best.block_cost, o_best.run_cost, o_best.num_ctas, o_best.merge, l2});
    }
    const Cand c = cands[ci];
    hbx_options o = b0;
    o.block_cost = c.block;
    o.run_cost = c.run;
    o.num_ctas = c.ctas;
    o.merge = c.merge;
    o.l2_keep_mb = c.l2;
    hbx_hmat *h = nullptr;
    int rc = hbx_create(st, nd, &o, &h);
    if (rc != HBX_OK) { rc_all = rc; continue; }
    auto launch = [&]() {
      return multi ? hbx_matmat(h, 1.0, static_cast<const float *>(x), 0.0, nullptr, y, s)
                   : hbx_matvec(h, 1.0, static_cast<const double *>(x), 0.0, nullptr, y, s);
    };
    for (int k = 0; k < 3 && rc == HBX_OK; ++k) rc = launch();
    cudaEventRecord(e0, s);
    for (int k = 0; k < reps && rc == HBX_OK; ++k) rc = launch();
    cudaEventRecord(e1, s);
    if (rc == HBX_OK) rc = hbx_sync(h, s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    hbx_destroy(h);
    if (rc != HBX_OK) { rc_all = rc; continue; }
    const double us = 1e3 * ms / reps;
    if (c.block == 0 && c.run == 0 && c.ctas == 0 && c.merge == 0 && c.l2 == 0) t_def = us;
    if (us < t_best) {
      t_best = us;
      o_best = o;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  cudaFree(x);
  cudaFree(y);
  if (t_best >= 1e30) return fail(rc_all != HBX_OK ? rc_all : HBX_ERR_INVALID, "hbx_autotune: no candidate ran");
  if (best) *best = o_best;
  if (best_us) *best_us = t_best;
  if (default_us) *default_us = t_def;
  return HBX_OK;
}

// The single-vector calls on a multi-RHS engine (its stream is laid out for
// the tensor-core product only).
static int single_rhs(const hbx_hmat *h, const char *where) {
  if (h && h->nrhs > 1) return fail(HBX_ERR_UNSUPPORTED, std::string(where) + ": a multi-RHS engine takes hbx_matmat only");
  return HBX_OK;
}

int hbx_matmat(hbx_hmat *h, double alpha, const float *X, double beta, const double *Yin, double *Y, void *stream) {
  if (!h || !X || !Y) return fail(HBX_ERR_INVALID, "hbx_matmat: NULL argument");
  if (h->nrhs != hbx::kNrhs) return fail(HBX_ERR_UNSUPPORTED, "hbx_matmat: not a multi-RHS engine (hbx_options.nrhs)");
  if (beta != 0.0 && !Yin) return fail(HBX_ERR_INVALID, "hbx_matmat: beta != 0 needs Yin");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  hbx::MatmatArgs a{};
  a.stream = h->d_stream;
  a.recs = h->d_recs;
  a.ctas = h->d_ctas;
  a.lite = h->d_lite;
  a.x = X;
  a.yin = Yin;
  a.y = Y;
  a.zbu = h->d_zbum;
  a.alpha = alpha;
  a.beta = beta;
  a.gbar = h->d_gbar;
  a.err = h->d_err;
  a.timeout_ns = h->timeout_ns;
  cudaError_t e = hbx::launch_matmat(a, h->num_ctas, s);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_matmat launch");
  return HBX_OK;
}

int hbx_matvec(hbx_hmat *h, double alpha, const double *x, double beta, const double *yin, double *y, void *stream) {
  if (int rc = single_rhs(h, "hbx_matvec")) return rc;
  if (!h || !x || !y) return fail(HBX_ERR_INVALID, "hbx_matvec: NULL argument");
  if (beta != 0.0 && !yin) return fail(HBX_ERR_INVALID, "hbx_matvec: beta != 0 needs yin");
  cudaError_t e = mv_launch(h, matvec_args(h, alpha, x, beta, yin, y), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_matvec launch");
  return HBX_OK;
}

// Allocation-free matvec.  Some callers cannot call cudaMalloc once they are
// running: a host code that has reserved the GPU's memory for its own pool
// (a later cudaMalloc finds no room) or a loop that must not stall (cudaFree
// synchronizes the whole device).  This variant launches the same kernel as
// hbx_matvec but takes its per-call scratch -- the V^T x segments (zbu) and
// the grid-barrier words -- from a fixed 1 MiB device array compiled into the
// library, so the call allocates nothing.  The array's address is looked up
// once per device, with that device current, on its first call (make that
// first call before any stream capture).
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[128] = {nullptr};

int hbx_matvec_noalloc(hbx_hmat *h, double alpha, const double *x, double beta, const double *yin, double *y,
                       void *stream) {
  if (!h || !x || !y) return fail(HBX_ERR_INVALID, "hbx_matvec_noalloc: NULL argument");
  if (int rc = single_rhs(h, "hbx_matvec_noalloc")) return rc;
  if (beta != 0.0 && !yin) return fail(HBX_ERR_INVALID, "hbx_matvec_noalloc: beta != 0 needs yin");
  if (h->plan.precision != hbx::kFP64)
    return fail(HBX_ERR_UNSUPPORTED, "hbx_matvec_noalloc: FP64 engines only (use hbx_matvec)");
  if (h->plan.zbu_len > hbx::kNoallocZbuMax)
    return fail(HBX_ERR_INVALID, "hbx_matvec_noalloc: the matrix needs " + std::to_string(h->plan.zbu_len) +
                                     " zbu doubles; the static scratch holds " +
                                     std::to_string(hbx::kNoallocZbuMax) + " (use hbx_matvec)");
  if (h->device < 0 || h->device >= 128) return fail(HBX_ERR_UNSUPPORTED, "hbx_matvec_noalloc: device ordinal");
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    base = g_noalloc_ptr[h->device];
    if (!base) {
      int cur = -1;
      cudaError_t e = cudaGetDevice(&cur);
      if (e == cudaSuccess && cur != h->device) e = cudaSetDevice(h->device);
      if (e == cudaSuccess) e = hbx::noalloc_scratch_address(&base);
      if (cur >= 0 && cur != h->device) cudaSetDevice(cur);
      if (e != cudaSuccess || !base) return cuda_fail(e, "hbx_matvec_noalloc: cudaGetSymbolAddress");
      g_noalloc_ptr[h->device] = base;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  // the barrier words must start at zero; zbu is written before it is read
  cudaError_t e = cudaMemsetAsync(base, 0, hbx::kNoallocCtlBytes, s);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_matvec_noalloc: clear barrier words");
  hbx::MatvecArgs a = matvec_args(h, alpha, x, beta, yin, y);
  a.gbar = reinterpret_cast<unsigned *>(base);
  a.zbu = reinterpret_cast<double *>(reinterpret_cast<char *>(base) + hbx::kNoallocCtlBytes);
  a.prof = nullptr;
  e = hbx::launch_matvec(a, h->num_ctas, s, h->plan.precision);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_matvec_noalloc launch");
  return HBX_OK;
}

int hbx_sync(hbx_hmat *h, void *stream) {
  if (!h) return fail(HBX_ERR_INVALID, "hbx_sync: NULL handle");
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_sync");
  return check_device_error(h, (cudaStream_t)stream);
}

int hbx_matvec_host(hbx_hmat *h, const double *zu, double *zau, int accumulate, double *kernel_seconds,
                    double *copy_seconds) {
  if (!h || !zu || !zau) return fail(HBX_ERR_INVALID, "hbx_matvec_host: NULL argument");
  if (int rc = single_rhs(h, "hbx_matvec_host")) return rc;
  int st = ensure_host_staging(h);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd, bytes = n * sizeof(double);
  cudaStream_t s = h->stream;
  const double t0 = now_s();
  HBX_CUDA(cudaMemcpyAsync(h->d_x, zu, bytes, cudaMemcpyHostToDevice, s));
  if (accumulate) HBX_CUDA(cudaMemcpyAsync(h->d_y, zau, bytes, cudaMemcpyHostToDevice, s));
  HBX_CUDA(cudaEventRecord(h->ev0, s));
  HBX_CUDA(mv_launch(h, matvec_args(h, 1.0, h->d_x, accumulate ? 1.0 : 0.0, h->d_y, h->d_y), s));
  HBX_CUDA(cudaEventRecord(h->ev1, s));
  HBX_CUDA(cudaMemcpyAsync(zau, h->d_y, bytes, cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  const double t1 = now_s();
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (kernel_seconds) *kernel_seconds += ms * 1e-3;
  if (copy_seconds) *copy_seconds += (t1 - t0) - ms * 1e-3;
  return check_device_error(h, s);
}

static hbx::BicgArgs bicg_args(hbx_hmat *h, const double *b, double *u, double tol, int max_iter) {
  const size_t n = (size_t)h->plan.nd;
  hbx::BicgArgs a{};
  a.stream = h->d_stream;
  a.recs = h->d_recs;
  a.ctas = h->d_ctas;
  a.lite = h->d_lite;
  a.atoms = h->d_atoms;
  a.zbu = h->d_zbu;
  a.zbu_len = h->plan.zbu_len;
  a.gbar = h->d_gbar;
  a.err = h->d_err;
  a.timeout_ns = h->timeout_ns;
  a.b = b;
  a.u = u;
  a.r = h->d_work;
  a.rh = h->d_work + n;
  a.p = h->d_work + 2 * n;
  a.ap = h->d_work + 3 * n;
  a.t = h->d_work + 4 * n;
  a.at = h->d_work + 5 * n;
  if (h->d_f32) {
    a.p32 = h->d_f32 + n;
    a.t32 = h->d_f32 + 2 * n;
    a.zbu32 = h->d_f32 + 3 * n;
  }
  a.part = h->d_part;
  a.state = h->d_state;
  a.hist = h->d_hist;
  a.prof = h->d_prof;
  a.tol = tol;
  a.max_iter = max_iter;
  a.keep_frac = h->keep_frac;
  return a;
}

// Captures `batch` iteration launches into one graph (re-captured when the
// vectors or the stopping parameters change).
static int get_graph(hbx_hmat *h, const hbx::BicgArgs &a, int batch) {
  const void *key[4] = {a.b, a.u, (const void *)(uintptr_t)a.max_iter, nullptr};
  double tolkey = a.tol;
  std::memcpy(&key[3], &tolkey, sizeof(double));
  if (h->graph && h->graph_batch == batch && std::memcmp(key, h->graph_key, sizeof(key)) == 0) return HBX_OK;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  cudaStream_t s = h->stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HBX_ERR_CUDA;
  for (int i = 0; i < batch; ++i) hbx::launch_bicg_iter(a, h->num_ctas, s, h->plan.precision);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess || !g) {
    cudaGetLastError();
    return HBX_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->graph = nullptr;
    return HBX_ERR_CUDA;
  }
  h->graph_batch = batch;
  std::memcpy(h->graph_key, key, sizeof(key));
  return HBX_OK;
}

// BiCGSTAB on device vectors b, u (u: x0 in / solution out), all on h->stream.
static int bicgstab_dev(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info) {
  if (int rc = single_rhs(h, "hbx_bicgstab")) return rc;
  const double tol = opts ? opts->tol : 1e-8;
  const int max_iter = opts ? opts->max_iter : 1000;
  const int verbose = opts ? opts->verbose : 0;
  int batch = (opts && opts->batch > 0) ? opts->batch : 8;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_bicgstab: bad tol or max_iter");
  int st = ensure_solver(h, max_iter);
  if (st != HBX_OK) return st;
  cudaStream_t s = h->stream;
  const hbx::BicgArgs a = bicg_args(h, b, u, tol, max_iter);
  HBX_CUDA(cudaEventRecord(h->ev0, s));
  // r = b - H u  (HACApK_SOLVER.c:562-573)
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, a.r), s));
  HBX_CUDA(hbx::launch_bicg_setup(a, h->num_ctas, s));
  const bool use_graph = get_graph(h, a, batch) == HBX_OK;
  int launched = 0;
  double iter_s = 0.0;
  for (;;) {
    HBX_CUDA(cudaEventRecord(h->ev3, s));
    if (use_graph) {
      HBX_CUDA(cudaGraphLaunch(h->graph, s));
    } else {
      for (int i = 0; i < batch; ++i) HBX_CUDA(hbx::launch_bicg_iter(a, h->num_ctas, s, h->plan.precision));
    }
    HBX_CUDA(cudaEventRecord(h->ev4, s));
    launched += batch;
    HBX_CUDA(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(hbx::BicgState), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    float bms = 0.f;
    cudaEventElapsedTime(&bms, h->ev3, h->ev4);
    iter_s += bms * 1e-3;
    if (h->h_state->done || launched > max_iter + batch) break;
    int derr = 0;
    HBX_CUDA(cudaMemcpy(&derr, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (derr) break;
  }
  HBX_CUDA(cudaEventRecord(h->ev1, s));
  const hbx::BicgState S = *h->h_state;
  // true residual ||b - H u|| (HACApK_SOLVER.c:737-746)
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, a.t), s));
  HBX_CUDA(hbx::launch_dot(a, a.t, a.t, hbx::kSlotAux, h->d_dot, h->num_ctas, s));
  double tr2 = 0.0;
  HBX_CUDA(cudaMemcpyAsync(&tr2, h->d_dot, sizeof(double), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  int dst = check_device_error(h, s);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->iterations = S.iter;
    info->status = dst != HBX_OK ? dst : S.status;
    info->bnorm = S.bnorm;
    info->relres = S.relres;
    info->true_relres = S.bnorm > 0 ? std::sqrt(tr2) / S.bnorm : std::sqrt(tr2);
    info->seconds = ms * 1e-3;
    info->iter_kernel_seconds = iter_s;
    info->iter_launches = launched;
    info->launches = launched + 5;  // r0 matvec, setup, residual matvec, two dot kernels
  }
  if (verbose > 0) {
    std::vector<double> hist(S.iter + 1, 0.0);
    if (S.iter > 0) cudaMemcpy(hist.data(), h->d_hist, S.iter * sizeof(double), cudaMemcpyDeviceToHost);
    hist[S.iter] = S.relres;
    std::printf("\n ** BICG (B200 persistent kernel) **\n");
    std::printf("\nOriginal relative residual norm = %.2e\n", hist[0]);
    for (int i = 1; i <= S.iter; ++i) std::printf(" %d: log10(zrnorm/bnorm)=%.2e\n", i, std::log10(hist[i]));
    std::printf("       BiCG        = %.5e\n", ms * 1e-3);
    std::printf(" resnorm=%.2e\n", std::sqrt(tr2));
    std::fflush(stdout);
  }
  if (dst != HBX_OK) return dst;
  if (!S.done) return fail(HBX_ERR_NOT_CONVERGED, "hbx_bicgstab: iteration limit");
  if (S.status != HBX_OK) return fail(S.status, std::string("hbx_bicgstab: ") + hbx_status_string(S.status));
  return HBX_OK;
}

int hbx_bicgstab(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info,
                 void *stream) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab: NULL argument");
  cudaStream_t us = (cudaStream_t)stream;
  HBX_CUDA(cudaEventRecord(h->ev2, us));
  HBX_CUDA(cudaStreamWaitEvent(h->stream, h->ev2, 0));
  int st = bicgstab_dev(h, b, u, opts, info);
  cudaEventRecord(h->ev2, h->stream);
  cudaStreamWaitEvent(us, h->ev2, 0);
  return st;
}

int hbx_bicgstab_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_host: NULL argument");
  const int max_iter = opts ? opts->max_iter : 1000;
  int st = ensure_solver(h, max_iter < 0 ? 0 : max_iter);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd, bytes = n * sizeof(double);
  double *db = h->d_work + 6 * n, *du = h->d_work + 7 * n;
  cudaStream_t s = h->stream;
  HBX_CUDA(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, s));
  HBX_CUDA(cudaMemcpyAsync(du, u, bytes, cudaMemcpyHostToDevice, s));
  st = bicgstab_dev(h, db, du, opts, info);
  cudaError_t e = cudaMemcpyAsync(u, du, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_bicgstab_host copy-out");
  return st;
}

// Pipelined BiCGSTAB of c_hacapk_bicgstab_cax_lfmtx_pipe_ (HACApK_SOLVER_PIPE.c:144-600)
// on device vectors, on h->stream: three products and k_pipe_init, then
// batches of steps (k_pipe_a, v = H z, k_pipe_b, t = H w) as one captured
// graph, the device state read back after each batch.
static int pipe_graph(hbx_hmat *h, const hbx::PipeVecs &v, int batch) {
  if (h->pgraph && h->pgraph_batch == batch && h->pgraph_key == v.u) return HBX_OK;
  if (h->pgraph) {
    cudaGraphExecDestroy(h->pgraph);
    h->pgraph = nullptr;
  }
  const size_t n = (size_t)h->plan.nd;
  cudaStream_t s = h->stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HBX_ERR_CUDA;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < batch && e == cudaSuccess; ++i) {
    hbx::MatvecArgs av = matvec_args(h, 1.0, v.z, 0.0, nullptr, v.v);
    av.skip = &h->d_pstate->done;
    hbx::MatvecArgs at = matvec_args(h, 1.0, v.w, 0.0, nullptr, v.t);
    at.skip = &h->d_pstate->done;
    e = hbx::pipe_launch_a(v, n, h->d_pstate, h->d_ppart, s);
    if (e == cudaSuccess) e = mv_launch(h, av, s);
    if (e == cudaSuccess) e = hbx::pipe_launch_b(v, n, h->d_pstate, h->d_ppart, h->d_phist, s);
    if (e == cudaSuccess) e = mv_launch(h, at, s);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return HBX_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&h->pgraph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->pgraph = nullptr;
    return HBX_ERR_CUDA;
  }
  h->pgraph_batch = batch;
  h->pgraph_key = v.u;
  return HBX_OK;
}

static int pipe_dev(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info) {
  if (int rc = single_rhs(h, "hbx_bicgstab_pipe")) return rc;
  const double tol = opts ? opts->tol : 1e-8;
  const int max_iter = opts ? opts->max_iter : 1000;
  const int verbose = opts ? opts->verbose : 0;
  const int batch = (opts && opts->batch > 0) ? opts->batch : 8;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_bicgstab_pipe: bad tol or max_iter");
  const size_t n = (size_t)h->plan.nd;
  if (!h->d_pipe) HBX_CUDA(dev_malloc(&h->d_pipe, (size_t)hbx::kPipeVecs * n * sizeof(double)));
  if (!h->d_pstate) {
    HBX_CUDA(dev_malloc(&h->d_pstate, sizeof(hbx::PipeState)));
    HBX_CUDA(cudaMemset(h->d_pstate, 0, sizeof(hbx::PipeState)));
  }
  if (!h->h_pstate) HBX_CUDA(cudaHostAlloc(&h->h_pstate, sizeof(hbx::PipeState), cudaHostAllocDefault));
  if (!h->d_ppart) HBX_CUDA(dev_malloc(&h->d_ppart, (size_t)hbx::gcr_dot_blocks(n) * hbx::kMaxDots * 2 * sizeof(double)));
  if (h->phist_cap < max_iter + 1) {
    if (h->pgraph) {  // the captured steps write the history being replaced
      cudaStreamSynchronize(h->stream);
      cudaGraphExecDestroy(h->pgraph);
      h->pgraph = nullptr;
    }
    cudaFree(h->d_phist);
    h->d_phist = nullptr;
    h->phist_cap = 0;
    HBX_CUDA(dev_malloc(&h->d_phist, (size_t)(max_iter + 1) * sizeof(double)));
    h->phist_cap = max_iter + 1;
  }
  double *V = h->d_pipe;
  hbx::PipeVecs v{b, u, V, V + n, V + 2 * n, V + 3 * n, V + 4 * n, V + 5 * n, V + 6 * n, V + 7 * n, V + 8 * n, V + 9 * n};
  cudaStream_t s = h->stream;
  HBX_CUDA(cudaEventRecord(h->ev0, s));
  // r = b - H u, r0 = r, w = H r, t = H w (HACApK_SOLVER_PIPE.c:283-356)
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, v.r), s));
  HBX_CUDA(mv_launch(h, matvec_args(h, 1.0, v.r, 0.0, nullptr, v.w), s));
  HBX_CUDA(mv_launch(h, matvec_args(h, 1.0, v.w, 0.0, nullptr, v.t), s));
  HBX_CUDA(hbx::pipe_launch_init(v, n, h->d_pstate, h->d_ppart, h->d_phist, tol, max_iter, s));
  HBX_CUDA(cudaMemcpyAsync(h->h_pstate, h->d_pstate, sizeof(hbx::PipeState), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  const bool use_graph = !h->h_pstate->done && pipe_graph(h, v, batch) == HBX_OK;
  int launched = 0;
  double iter_s = 0.0;
  while (!h->h_pstate->done && launched <= max_iter + batch) {
    HBX_CUDA(cudaEventRecord(h->ev3, s));
    if (use_graph) {
      HBX_CUDA(cudaGraphLaunch(h->pgraph, s));
    } else {
      for (int i = 0; i < batch; ++i) {
        hbx::MatvecArgs av = matvec_args(h, 1.0, v.z, 0.0, nullptr, v.v);
        av.skip = &h->d_pstate->done;
        hbx::MatvecArgs at = matvec_args(h, 1.0, v.w, 0.0, nullptr, v.t);
        at.skip = &h->d_pstate->done;
        HBX_CUDA(hbx::pipe_launch_a(v, n, h->d_pstate, h->d_ppart, s));
        HBX_CUDA(mv_launch(h, av, s));
        HBX_CUDA(hbx::pipe_launch_b(v, n, h->d_pstate, h->d_ppart, h->d_phist, s));
        HBX_CUDA(mv_launch(h, at, s));
      }
    }
    HBX_CUDA(cudaEventRecord(h->ev4, s));
    launched += batch;
    HBX_CUDA(cudaMemcpyAsync(h->h_pstate, h->d_pstate, sizeof(hbx::PipeState), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    float bms = 0.f;
    cudaEventElapsedTime(&bms, h->ev3, h->ev4);
    iter_s += bms * 1e-3;
    int derr = 0;
    HBX_CUDA(cudaMemcpy(&derr, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (derr) break;
  }
  HBX_CUDA(cudaEventRecord(h->ev1, s));
  const hbx::PipeState S = *h->h_pstate;
  // true residual ||b - H u||, in v.v (no longer needed)
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, v.v), s));
  const double *xs[1] = {v.v}, *ys[1] = {v.v};
  HBX_CUDA(hbx::gcr_launch_dots(1, xs, ys, n, h->d_ppart, h->d_pipe + 8 * n, s));  // into q (free now)
  double tr2 = 0.0;
  HBX_CUDA(cudaMemcpyAsync(&tr2, h->d_pipe + 8 * n, sizeof(double), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  int dst = check_device_error(h, s);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->iterations = S.step;
    info->status = dst != HBX_OK ? dst : S.status;
    info->bnorm = S.bnorm;
    info->relres = S.relres;
    info->true_relres = S.bnorm > 0 ? std::sqrt(tr2) / S.bnorm : std::sqrt(tr2);
    info->seconds = ms * 1e-3;
    info->iter_kernel_seconds = iter_s;
    info->iter_launches = 4 * launched;
    info->launches = 4 * launched + 7;  // 3 setup products, init, residual product, two dot kernels
  }
  if (verbose > 0) {
    std::vector<double> hist(S.step + 1, 0.0);
    cudaMemcpy(hist.data(), h->d_phist, (S.step + 1) * sizeof(double), cudaMemcpyDeviceToHost);
    std::printf("\n ** pipelined BICG (version 1) (B200 kernels) **\n");
    std::printf("\nOriginal relative residual norm = %.2e\n", hist[0]);
    for (int i = 1; i <= S.step; ++i) std::printf(" %d: log10(zrnorm/bnorm)=%.2e\n", i, std::log10(hist[i]));
    std::printf("       BiCG        = %.5e\n", ms * 1e-3);
    std::fflush(stdout);
  }
  if (dst != HBX_OK) return dst;
  if (!S.done) return fail(HBX_ERR_NOT_CONVERGED, "hbx_bicgstab_pipe: iteration limit");
  if (S.status != HBX_OK) return fail(S.status, std::string("hbx_bicgstab_pipe: ") + hbx_status_string(S.status));
  return HBX_OK;
}

int hbx_bicgstab_pipe(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info,
                      void *stream) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_pipe: NULL argument");
  cudaStream_t us = (cudaStream_t)stream;
  HBX_CUDA(cudaEventRecord(h->ev2, us));
  HBX_CUDA(cudaStreamWaitEvent(h->stream, h->ev2, 0));
  int st = pipe_dev(h, b, u, opts, info);
  cudaEventRecord(h->ev2, h->stream);
  cudaStreamWaitEvent(us, h->ev2, 0);
  return st;
}

int hbx_bicgstab_pipe_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts,
                           hbx_solve_info *info) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_pipe_host: NULL argument");
  int st = ensure_solver(h, 0);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd, bytes = n * sizeof(double);
  double *db = h->d_work + 6 * n, *du = h->d_work + 7 * n;
  cudaStream_t s = h->stream;
  HBX_CUDA(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, s));
  HBX_CUDA(cudaMemcpyAsync(du, u, bytes, cudaMemcpyHostToDevice, s));
  st = pipe_dev(h, db, du, opts, info);
  cudaError_t e = cudaMemcpyAsync(u, du, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_bicgstab_pipe_host copy-out");
  return st;
}

// GCR(m) of HACApK_gcrm_lfmtx (m_HACApK_solve.f90:506-571) on device vectors,
// on h->stream: r = b - H u, k_gcr_init, A p_0, k_gcr_alpha0, then whole
// restart cycles (per step: k_gcr_update, A r, k_gcr_proj + k_gcr_orth) as
// one captured graph, the device state read back after each graph.
static void gcr_step(hbx_hmat *h, const hbx::GcrVecs &v, int m, int in, cudaStream_t s, cudaError_t &e) {
  const size_t n = (size_t)h->plan.nd;
  const int ik = (in - 1) % m, ikn = in % m;
  if (e == cudaSuccess) e = hbx::gcr_launch_update(v, n, ik, h->d_gcrs, h->d_gcrpart, s);
  hbx::MatvecArgs a = matvec_args(h, 1.0, v.r, 0.0, nullptr, v.ar);
  a.skip = &h->d_gcrs->done;
  if (e == cudaSuccess) e = mv_launch(h, a, s);
  if (e == cudaSuccess) e = hbx::gcr_launch_orth(v, n, ik, ikn, h->d_gcrs, h->d_gcrpart, s);
}

static int gcr_graph(hbx_hmat *h, const hbx::GcrVecs &v, int m, int cycles) {
  if (h->ggraph && h->ggraph_m == m && h->ggraph_cycles == cycles && h->ggraph_key == v.u) return HBX_OK;
  if (h->ggraph) {
    cudaGraphExecDestroy(h->ggraph);
    h->ggraph = nullptr;
  }
  cudaStream_t s = h->stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HBX_ERR_CUDA;
  cudaError_t e = cudaSuccess;
  for (int in = 1; in <= m * cycles; ++in) gcr_step(h, v, m, in, s, e);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return HBX_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&h->ggraph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->ggraph = nullptr;
    return HBX_ERR_CUDA;
  }
  h->ggraph_m = m;
  h->ggraph_cycles = cycles;
  h->ggraph_key = v.u;
  return HBX_OK;
}

static int gcr_dev(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info) {
  if (int rc = single_rhs(h, "hbx_gcr")) return rc;
  const double tol = opts ? opts->tol : 1e-8;
  const int mstep = opts ? opts->max_iter : 1000;
  const int m = (opts && opts->restart > 0) ? opts->restart : 8;
  if (mstep < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_gcr: bad tol or max_iter");
  if (m > hbx::kMaxDots) return fail(HBX_ERR_INVALID, "hbx_gcr: restart length above " + std::to_string(hbx::kMaxDots));
  const size_t n = (size_t)h->plan.nd;
  if (h->gcr_m < m) {
    cudaFree(h->d_gcr);
    h->d_gcr = nullptr;
    h->gcr_m = 0;
    HBX_CUDA(dev_malloc(&h->d_gcr, (2 + 2 * (size_t)m) * n * sizeof(double)));
    h->gcr_m = m;
    if (h->ggraph) {
      cudaGraphExecDestroy(h->ggraph);
      h->ggraph = nullptr;
    }
  }
  if (!h->d_gcrs) {
    HBX_CUDA(dev_malloc(&h->d_gcrs, sizeof(hbx::GcrState)));
    HBX_CUDA(cudaMemset(h->d_gcrs, 0, sizeof(hbx::GcrState)));
  }
  if (!h->h_gcrs) HBX_CUDA(cudaHostAlloc(&h->h_gcrs, sizeof(hbx::GcrState), cudaHostAllocDefault));
  if (!h->d_gcrpart)
    HBX_CUDA(dev_malloc(&h->d_gcrpart, (size_t)hbx::gcr_dot_blocks(n) * hbx::kMaxDots * 2 * sizeof(double)));
  cudaStream_t s = h->stream;
  const size_t slots = (size_t)h->gcr_m;  // the workspace holds gcr_m >= m slots of p, then of A p
  hbx::GcrVecs v{b, u, h->d_gcr, h->d_gcr + n, h->d_gcr + 2 * n, h->d_gcr + (2 + slots) * n};
  HBX_CUDA(cudaEventRecord(h->ev0, s));
  // zr = b - H u; zp(1) = zr; the first stop test; zap(1) = H zp(1); alpha
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, v.r), s));
  HBX_CUDA(hbx::gcr_launch_init(v, n, h->d_gcrs, h->d_gcrpart, tol, mstep, s));
  hbx::MatvecArgs a0 = matvec_args(h, 1.0, v.p, 0.0, nullptr, v.ap);
  a0.skip = &h->d_gcrs->done;
  HBX_CUDA(mv_launch(h, a0, s));
  HBX_CUDA(hbx::gcr_launch_alpha0(v, n, h->d_gcrs, h->d_gcrpart, s));
  HBX_CUDA(cudaMemcpyAsync(h->h_gcrs, h->d_gcrs, sizeof(hbx::GcrState), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  // steps per graph: whole cycles, at least 8 steps
  const int cycles = (8 + m - 1) / m;
  const bool use_graph = !h->h_gcrs->done && gcr_graph(h, v, m, cycles) == HBX_OK;
  int launched = 0;
  while (!h->h_gcrs->done && launched <= mstep + m * cycles) {
    if (use_graph) {
      HBX_CUDA(cudaGraphLaunch(h->ggraph, s));
    } else {
      cudaError_t e = cudaSuccess;
      for (int in = 1; in <= m * cycles; ++in) gcr_step(h, v, m, in, s, e);
      HBX_CUDA(e);
    }
    launched += m * cycles;
    HBX_CUDA(cudaMemcpyAsync(h->h_gcrs, h->d_gcrs, sizeof(hbx::GcrState), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    int derr = 0;
    HBX_CUDA(cudaMemcpy(&derr, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (derr) break;
  }
  HBX_CUDA(cudaEventRecord(h->ev1, s));
  const hbx::GcrState S = *h->h_gcrs;
  // true residual ||b - H u|| in A r (free now)
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, v.ar), s));
  const double *xs[1] = {v.ar}, *ys[1] = {v.ar};
  double *out = v.p;  // the search directions are no longer needed
  HBX_CUDA(hbx::gcr_launch_dots(1, xs, ys, n, h->d_gcrpart, out, s));
  double tr2 = 0.0;
  HBX_CUDA(cudaMemcpyAsync(&tr2, out, sizeof(double), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  int dst = check_device_error(h, s);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->iterations = S.step;
    info->status = dst != HBX_OK ? dst : S.status;
    info->bnorm = S.bnorm;
    info->relres = S.relres;
    info->true_relres = S.bnorm > 0 ? std::sqrt(tr2) / S.bnorm : std::sqrt(tr2);
    info->seconds = ms * 1e-3;
    info->iter_launches = 4 * launched;
    info->launches = 4 * launched + 7;
  }
  if (dst != HBX_OK) return dst;
  if (!S.done) return fail(HBX_ERR_NOT_CONVERGED, "hbx_gcr: iteration limit");
  if (S.status != HBX_OK) return fail(S.status, std::string("hbx_gcr: ") + hbx_status_string(S.status));
  return HBX_OK;
}

int hbx_gcr(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info, void *stream) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_gcr: NULL argument");
  cudaStream_t us = (cudaStream_t)stream;
  HBX_CUDA(cudaEventRecord(h->ev2, us));
  HBX_CUDA(cudaStreamWaitEvent(h->stream, h->ev2, 0));
  int st = gcr_dev(h, b, u, opts, info);
  cudaEventRecord(h->ev2, h->stream);
  cudaStreamWaitEvent(us, h->ev2, 0);
  return st;
}

int hbx_gcr_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_gcr_host: NULL argument");
  int st = ensure_solver(h, 0);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd, bytes = n * sizeof(double);
  double *db = h->d_work + 6 * n, *du = h->d_work + 7 * n;
  cudaStream_t s = h->stream;
  HBX_CUDA(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, s));
  HBX_CUDA(cudaMemcpyAsync(du, u, bytes, cudaMemcpyHostToDevice, s));
  st = gcr_dev(h, db, du, opts, info);
  cudaError_t e = cudaMemcpyAsync(u, du, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_gcr_host copy-out");
  return st;
}

// Mixed-precision solve: FP64 residuals on `h`, inner BiCGSTAB on `hl`, all
// on hl's stream.  The inner solve's target is relative to the current
// residual; the last one is asked for no more than the outer tolerance needs.
static int refined_dev(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                       hbx_solve_info *info) {
  if (int rc = single_rhs(h, "hbx_bicgstab_refined")) return rc;
  if (int rc = single_rhs(hl, "hbx_bicgstab_refined")) return rc;
  const double tol = opts ? opts->tol : 1e-8;
  const int max_iter = opts ? opts->max_iter : 1000;
  const double floor_tol = (opts && opts->inner_tol > 0.0) ? opts->inner_tol : 1e-6;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_bicgstab_refined: bad tol or max_iter");
  int st = ensure_solver(hl, max_iter);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd;
  if (!hl->d_refine) HBX_CUDA(dev_malloc(&hl->d_refine, 2 * n * sizeof(double)));
  double *r = hl->d_refine, *d = hl->d_refine + n;
  cudaStream_t s = hl->stream;
  const hbx::BicgArgs a = bicg_args(hl, b, u, tol, max_iter);
  auto dot = [&](const double *x, const double *y, double &out) -> int {
    HBX_CUDA(hbx::launch_dot(a, x, y, hbx::kSlotAux, hl->d_dot, hl->num_ctas, s));
    HBX_CUDA(cudaMemcpyAsync(&out, hl->d_dot, sizeof(double), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    return HBX_OK;
  };
  cudaEvent_t e0 = h->ev0, e1 = h->ev1;
  HBX_CUDA(cudaEventRecord(e0, s));
  double bb = 0.0;
  if ((st = dot(b, b, bb)) != HBX_OK) return st;
  const double bnorm = std::sqrt(bb);
  int inner_total = 0, outer = 0, launches = 1, status = HBX_ERR_NOT_CONVERGED;
  double relres = 1.0, iter_s = 0.0;
  for (;;) {
    HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, r), s));
    double rr = 0.0;
    if ((st = dot(r, r, rr)) != HBX_OK) return st;
    launches += 3;
    relres = bnorm > 0.0 ? std::sqrt(rr) / bnorm : std::sqrt(rr);
    if (!std::isfinite(relres)) { status = HBX_ERR_BREAKDOWN; break; }
    if (relres < tol) { status = HBX_OK; break; }
    if (inner_total >= max_iter || outer >= 64) break;
    HBX_CUDA(cudaMemsetAsync(d, 0, n * sizeof(double), s));
    hbx_solve_opts io{};
    io.tol = std::max(floor_tol, 0.5 * tol / relres);
    io.max_iter = max_iter - inner_total;
    io.batch = opts ? opts->batch : 0;
    hbx_solve_info ii{};
    int ist = bicgstab_dev(hl, r, d, &io, &ii);
    inner_total += ii.iterations;
    iter_s += ii.iter_kernel_seconds;
    launches += ii.launches;
    ++outer;
    if (ist != HBX_OK && ist != HBX_ERR_NOT_CONVERGED && ist != HBX_ERR_BREAKDOWN) return ist;
    if (ii.iterations == 0 && ist != HBX_OK) { status = ist; break; }
    HBX_CUDA(hbx::launch_axpy(1.0, d, u, n, s));
    ++launches;
  }
  HBX_CUDA(cudaEventRecord(e1, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->iterations = inner_total;
    info->outer = outer;
    info->status = status;
    info->bnorm = bnorm;
    info->relres = relres;
    info->true_relres = relres;
    info->seconds = ms * 1e-3;
    info->iter_kernel_seconds = iter_s;
    info->launches = launches;
  }
  if (status != HBX_OK) return fail(status, std::string("hbx_bicgstab_refined: ") + hbx_status_string(status));
  return check_device_error(hl, s);
}

int hbx_bicgstab_refined(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                         hbx_solve_info *info, void *stream) {
  if (!h || !hl || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_refined: NULL argument");
  if (h->plan.nd != hl->plan.nd || h->transposed != hl->transposed || h->device != hl->device)
    return fail(HBX_ERR_INVALID, "hbx_bicgstab_refined: h and hl must hold the same operator on one device");
  cudaStream_t us = (cudaStream_t)stream;
  HBX_CUDA(cudaEventRecord(hl->ev2, us));
  HBX_CUDA(cudaStreamWaitEvent(hl->stream, hl->ev2, 0));
  int st = refined_dev(h, hl, b, u, opts, info);
  cudaEventRecord(hl->ev2, hl->stream);
  cudaStreamWaitEvent(us, hl->ev2, 0);
  return st;
}

int hbx_bicgstab_refined_host(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                              hbx_solve_info *info) {
  if (!h || !hl || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_refined_host: NULL argument");
  if (h->plan.nd != hl->plan.nd || h->transposed != hl->transposed || h->device != hl->device)
    return fail(HBX_ERR_INVALID, "hbx_bicgstab_refined: h and hl must hold the same operator on one device");
  const int max_iter = opts ? opts->max_iter : 1000;
  int st = ensure_solver(hl, max_iter < 0 ? 0 : max_iter);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)hl->plan.nd, bytes = n * sizeof(double);
  double *db = hl->d_work + 6 * n, *du = hl->d_work + 7 * n;
  cudaStream_t s = hl->stream;
  HBX_CUDA(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, s));
  HBX_CUDA(cudaMemcpyAsync(du, u, bytes, cudaMemcpyHostToDevice, s));
  st = refined_dev(h, hl, db, du, opts, info);
  cudaError_t e = cudaMemcpyAsync(u, du, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_bicgstab_refined_host copy-out");
  return st;
}

// dJ/dg for J = 0.5 ||sigma - sigma_t||^2, H sigma = g: the forward solve,
// then the adjoint solve H^T lambda = sigma - sigma_t on the transposed engine.
int hbx_gradient_host(hbx_hmat *h, hbx_hmat *ht, const double *g, const double *sigma_t, double *sigma,
                      double *grad, double *J, const hbx_solve_opts *opts, hbx_solve_info *fwd,
                      hbx_solve_info *adj) {
  if (!h || !ht || !g || !sigma_t || !sigma || !grad) return fail(HBX_ERR_INVALID, "hbx_gradient_host: NULL argument");
  if (int rc = single_rhs(h, "hbx_gradient_host")) return rc;
  if (int rc = single_rhs(ht, "hbx_gradient_host")) return rc;
  if (h->transposed || !ht->transposed)
    return fail(HBX_ERR_INVALID, "hbx_gradient_host: h must hold H and ht must hold H^T (hbx_options.transpose)");
  if (h->plan.nd != ht->plan.nd) return fail(HBX_ERR_INVALID, "hbx_gradient_host: h and ht differ in size");
  const size_t n = (size_t)h->plan.nd;
  std::fill(sigma, sigma + n, 0.0);
  int st = hbx_bicgstab_host(h, g, sigma, opts, fwd);
  if (st != HBX_OK) return st;
  std::vector<double> d(n);
  double j = 0.0;
  for (size_t i = 0; i < n; ++i) {
    d[i] = sigma[i] - sigma_t[i];
    j += d[i] * d[i];
  }
  if (J) *J = 0.5 * j;
  std::fill(grad, grad + n, 0.0);
  return hbx_bicgstab_host(ht, d.data(), grad, opts, adj);
}

// ------------------------------------------------------------------------
// HACApK drop-in entry points
// ------------------------------------------------------------------------

static hbx_hmat *lookup(const stc_HACApK_leafmtxp *st) {
  std::lock_guard<std::mutex> lk(g_table_mu);
  auto it = g_table.find(st);
  return it == g_table.end() ? nullptr : it->second;
}

static hbx_hmat *create_for(stc_HACApK_leafmtxp *st, int nd) {
  hbx_hmat *h = nullptr;
  int rc = hbx_create(st, nd, nullptr, &h);
  if (rc != HBX_OK) {
    std::fprintf(stderr, "!!!! hacapk_b200: setup failed: %s (%s)\n", hbx_status_string(rc), hbx_last_error());
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_table_mu);
  auto it = g_table.find(st);
  if (it != g_table.end()) hbx_destroy(it->second);
  g_table[st] = h;
  return h;
}

static void release_for(stc_HACApK_leafmtxp *st) {
  hbx_hmat *h = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_table.find(st);
    if (it == g_table.end()) return;
    h = it->second;
    g_table.erase(it);
  }
  hbx_destroy(h);
}

void magma_init_(void) { cudaFree(nullptr); }

void magma_finalize_(void) {}

// ---- multi-RHS BiCGSTAB in FP64 iterative refinement ----------------------
namespace {

struct MrPinned {
  hbx::MrScal sc[hbx::kNrhs];
  double norm[hbx::kNrhs];
  double thresh[hbx::kNrhs];
  int mask[hbx::kNrhs];
  int any;
};

// Each buffer is tested on its own, so a call after a failed allocation
// completes the set instead of running on a null pointer.
int ensure_mr_workspace(hbx_hmat *hm) {
  const size_t n = (size_t)hm->plan.nd * hbx::kNrhs;
  if (!hm->d_mrv) HBX_CUDA(dev_malloc(&hm->d_mrv, 10 * n * sizeof(double)));
  if (!hm->d_mr32) HBX_CUDA(dev_malloc(&hm->d_mr32, n * sizeof(float)));
  if (!hm->d_mrpart)
    HBX_CUDA(dev_malloc(&hm->d_mrpart, (size_t)hbx::mr_row_blocks(hm->plan.nd) * 2 * hbx::kNrhs * sizeof(double)));
  if (!hm->d_mrsc) HBX_CUDA(dev_malloc(&hm->d_mrsc, hbx::kNrhs * sizeof(hbx::MrScal)));
  if (!hm->d_mrint) HBX_CUDA(dev_malloc(&hm->d_mrint, (1 + hbx::kNrhs) * sizeof(int)));
  if (!hm->d_mrdbl) HBX_CUDA(dev_malloc(&hm->d_mrdbl, 2 * hbx::kNrhs * sizeof(double)));
  if (!hm->h_mrpin) HBX_CUDA(cudaMallocHost(&hm->h_mrpin, sizeof(MrPinned)));
  return HBX_OK;
}

cudaError_t mr_matmat(void *ctx, const float *x, double *y, cudaStream_t s) {
  hbx_hmat *hm = static_cast<hbx_hmat *>(ctx);
  hbx::MatmatArgs a{};
  a.stream = hm->d_stream;
  a.recs = hm->d_recs;
  a.ctas = hm->d_ctas;
  a.lite = hm->d_lite;
  a.x = x;
  a.y = y;
  a.zbu = hm->d_zbum;
  a.alpha = 1.0;
  a.beta = 0.0;
  a.gbar = hm->d_gbar;
  a.err = hm->d_err;
  a.timeout_ns = hm->timeout_ns;
  return hbx::launch_matmat(a, hm->num_ctas, s);
}

}  // namespace

int hbx_bicgstab_multi(hbx_hmat *h, hbx_hmat *hm, const double *B, double *U, const hbx_solve_opts *opts,
                       hbx_solve_info *info, void *stream) {
  if (!h || !hm || !B || !U) return fail(HBX_ERR_INVALID, "hbx_bicgstab_multi: NULL argument");
  if (int rc = single_rhs(h, "hbx_bicgstab_multi")) return rc;
  if (hm->nrhs != hbx::kNrhs) return fail(HBX_ERR_UNSUPPORTED, "hbx_bicgstab_multi: hm is not a multi-RHS engine");
  if (h->plan.precision != hbx::kFP64) return fail(HBX_ERR_UNSUPPORTED, "hbx_bicgstab_multi: h must hold FP64 factors");
  if (h->plan.nd != hm->plan.nd || h->transposed != hm->transposed || h->device != hm->device)
    return fail(HBX_ERR_INVALID, "hbx_bicgstab_multi: h and hm differ (size, orientation or device)");
  const double tol = opts ? opts->tol : 1e-8;
  const int max_iter = opts ? opts->max_iter : 1000;
  const double floor_tol = (opts && opts->inner_tol > 0.0) ? opts->inner_tol : 1e-3;
  const int batch = (opts && opts->batch > 0) ? opts->batch : 4;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_bicgstab_multi: bad tol or max_iter");
  int st = ensure_mr_workspace(hm);
  if (st != HBX_OK) return st;
  const int nd = h->plan.nd;
  const size_t n = (size_t)nd * hbx::kNrhs;
  double *r = hm->d_mrv, *rh = r + n, *p = rh + n, *ap = p + n, *t = ap + n, *at = t + n, *x = at + n, *R = x + n,
         *T1 = R + n, *T2 = T1 + n;
  double *d_thr = hm->d_mrdbl, *d_norm = hm->d_mrdbl + hbx::kNrhs;
  int *d_any = hm->d_mrint, *d_mask = hm->d_mrint + 1;
  MrPinned *pin = static_cast<MrPinned *>(hm->h_mrpin);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto norms = [&](const double *v) -> int {  // pin->norm[j] = ||v_j||^2
    HBX_CUDA(hbx::mr_launch_dots(1, nd, v, v, nullptr, nullptr, hm->d_mrpart, s));
    HBX_CUDA(hbx::mr_launch_colsum(nd, hm->d_mrpart, d_norm, s));
    HBX_CUDA(cudaMemcpyAsync(pin->norm, d_norm, sizeof(pin->norm), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    return HBX_OK;
  };
  HBX_CUDA(cudaEventRecord(hm->ev0, s));
  if ((st = norms(B)) != HBX_OK) return st;
  double bnorm[hbx::kNrhs], relres[hbx::kNrhs];
  int done[hbx::kNrhs], status[hbx::kNrhs], iters[hbx::kNrhs];
  for (int j = 0; j < hbx::kNrhs; ++j) {
    bnorm[j] = std::sqrt(pin->norm[j]);
    relres[j] = 1.0;
    done[j] = 0;
    status[j] = HBX_ERR_NOT_CONVERGED;
    iters[j] = 0;
  }
  int outer = 0, launches = 1, steps = 0;
  for (;;) {
    // R = B - H U, FP64: one product per right-hand side still running whose
    // U is not zero (x0 = 0 makes the first residual B itself)
    if ((st = norms(U)) != HBX_OK) return st;
    HBX_CUDA(hbx::mr_launch_transpose(nd, hbx::kNrhs, U, T1, s));
    for (int j = 0; j < hbx::kNrhs; ++j) {
      if (done[j]) continue;
      if (pin->norm[j] == 0.0) HBX_CUDA(cudaMemsetAsync(T2 + (size_t)j * nd, 0, (size_t)nd * sizeof(double), s));
      else HBX_CUDA(mv_launch(h, matvec_args(h, 1.0, T1 + (size_t)j * nd, 0.0, nullptr, T2 + (size_t)j * nd), s));
    }
    HBX_CUDA(hbx::mr_launch_resid(nd, B, T2, R, s));
    if ((st = norms(R)) != HBX_OK) return st;
    if ((st = check_device_error(h, s)) != HBX_OK) return st;
    launches += 4 + hbx::kNrhs;
    int running = 0, max_done_iters = 0;
    for (int j = 0; j < hbx::kNrhs; ++j) {
      if (done[j]) continue;
      const double rn = std::sqrt(pin->norm[j]);
      relres[j] = bnorm[j] > 0.0 ? rn / bnorm[j] : rn;
      if (!std::isfinite(relres[j])) { done[j] = 1; status[j] = HBX_ERR_BREAKDOWN; continue; }
      if (relres[j] < tol) { done[j] = 1; status[j] = HBX_OK; continue; }
      if (iters[j] >= max_iter || outer >= 64) { done[j] = 1; continue; }
      max_done_iters = std::max(max_done_iters, iters[j]);
      ++running;
    }
    if (running == 0) break;
    for (int j = 0; j < hbx::kNrhs; ++j) {
      pin->mask[j] = !done[j];
      pin->thresh[j] = done[j] ? 0.0 : std::max(floor_tol, 0.5 * tol / relres[j]) * relres[j] * (bnorm[j] > 0.0 ? bnorm[j] : 1.0);
    }
    HBX_CUDA(cudaMemcpyAsync(d_thr, pin->thresh, sizeof(pin->thresh), cudaMemcpyHostToDevice, s));
    HBX_CUDA(cudaMemcpyAsync(d_mask, pin->mask, sizeof(pin->mask), cudaMemcpyHostToDevice, s));
    HBX_CUDA(hbx::mr_launch_setup(nd, R, r, rh, p, ap, x, s));
    HBX_CUDA(hbx::mr_launch_dots(1, nd, r, r, nullptr, nullptr, hm->d_mrpart, s));
    HBX_CUDA(hbx::mr_launch_init(nd, hm->d_mrpart, d_thr, d_mask, hm->d_mrsc, d_any, s));
    launches += 3;
    hbx::MrStep a{};
    a.nd = nd;
    a.max_iter = std::max(1, max_iter - max_done_iters);
    a.sc = hm->d_mrsc;
    a.any_active = d_any;
    a.r = r; a.rh = rh; a.p = p; a.ap = ap; a.t = t; a.at = at; a.x = x; a.part = hm->d_mrpart;
    a.f32 = hm->d_mr32;
    a.matmat = mr_matmat;
    a.ctx = hm;
    for (int k = 0; k < a.max_iter; k += batch) {
      HBX_CUDA(cudaMemcpyAsync(&pin->any, d_any, sizeof(int), cudaMemcpyDeviceToHost, s));
      HBX_CUDA(cudaStreamSynchronize(s));
      if (!pin->any) break;
      for (int b = 0; b < batch; ++b) HBX_CUDA(hbx::mr_launch_step(a, s));
      launches += 10 * batch;
      steps += batch;
    }
    HBX_CUDA(cudaMemcpyAsync(pin->sc, hm->d_mrsc, sizeof(pin->sc), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(hbx::mr_launch_add(nd, d_mask, x, U, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    if ((st = check_device_error(hm, s)) != HBX_OK) return st;
    ++launches;
    for (int j = 0; j < hbx::kNrhs; ++j) {
      if (done[j]) continue;
      iters[j] += pin->sc[j].iters;
      // an inner solve that broke down before its first step leaves nothing to refine
      if (pin->sc[j].iters == 0 && pin->sc[j].status == HBX_ERR_BREAKDOWN) { done[j] = 1; status[j] = HBX_ERR_BREAKDOWN; }
    }
    ++outer;
  }
  HBX_CUDA(cudaEventRecord(hm->ev1, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, hm->ev0, hm->ev1);
  int worst = HBX_OK;
  for (int j = 0; j < hbx::kNrhs; ++j) {
    if (status[j] != HBX_OK && worst == HBX_OK) worst = status[j];
    if (info) {
      hbx_solve_info &I = info[j];
      std::memset(&I, 0, sizeof(I));
      I.iterations = iters[j];
      I.outer = outer;
      I.status = status[j];
      I.bnorm = bnorm[j];
      I.relres = relres[j];
      I.true_relres = relres[j];
      I.seconds = ms * 1e-3;
      I.launches = launches;
      I.iter_launches = steps;
    }
  }
  if (worst != HBX_OK) return fail(worst, std::string("hbx_bicgstab_multi: ") + hbx_status_string(worst));
  return HBX_OK;
}


int hbx_bicgstab_multi_host(hbx_hmat *h, hbx_hmat *hm, const double *B, double *U, const hbx_solve_opts *opts,
                            hbx_solve_info *info) {
  if (!h || !hm || !B || !U) return fail(HBX_ERR_INVALID, "hbx_bicgstab_multi_host: NULL argument");
  if (hm->nrhs != hbx::kNrhs) return fail(HBX_ERR_UNSUPPORTED, "hbx_bicgstab_multi_host: hm is not a multi-RHS engine");
  int st = ensure_mr_workspace(hm);
  if (st != HBX_OK) return st;
  const size_t bytes = (size_t)hm->plan.nd * hbx::kNrhs * sizeof(double);
  double *dB = nullptr, *dU = nullptr;
  HBX_CUDA(dev_malloc(&dB, 2 * bytes));
  dU = dB + (size_t)hm->plan.nd * hbx::kNrhs;
  cudaStream_t s = hm->stream;
  cudaError_t e = cudaMemcpyAsync(dB, B, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dU, U, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) { cudaFree(dB); return cuda_fail(e, "hbx_bicgstab_multi_host upload"); }
  st = hbx_bicgstab_multi(h, hm, dB, dU, opts, info, s);
  e = cudaMemcpyAsync(U, dU, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dB);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_bicgstab_multi_host download");
  return st;
}


// ---- batched BiCGSTAB over the instances of a block-diagonal engine -----------
namespace {

// HBX_STREAM_ALL=1 makes the batched solves stream every instance's bytes
// every step (the per-instance chunk skipping off), for comparisons.
bool skip_disabled() {
  const char *v = std::getenv("HBX_STREAM_ALL");
  return v && std::atoi(v) != 0;
}

cudaError_t bt_matvec(void *ctx, const double *x, double *y, cudaStream_t s) {
  hbx_hmat *h = static_cast<hbx_hmat *>(ctx);
  return mv_launch(h, matvec_args(h, 1.0, x, 0.0, nullptr, y), s);
}

// A plain engine is one instance.  Its tables are published (inst_off set)
// only once both are on the device, and each work buffer is tested on its
// own, so a call after a failed allocation never runs on a null pointer.
int ensure_bt_workspace(hbx_hmat *h, int count) {
  const size_t n = (size_t)h->plan.nd;
  if (h->inst_off.empty()) {
    const int off[2] = {0, h->plan.nd};
    if (!h->d_inst_off) HBX_CUDA(dev_malloc(&h->d_inst_off, 2 * sizeof(int)));
    if (!h->d_rinst) HBX_CUDA(dev_malloc(&h->d_rinst, n * sizeof(int)));
    HBX_CUDA(cudaMemcpy(h->d_inst_off, off, 2 * sizeof(int), cudaMemcpyHostToDevice));
    HBX_CUDA(cudaMemset(h->d_rinst, 0, n * sizeof(int)));
    h->inst_off.assign(off, off + 2);
  }
  if (!h->d_btv) HBX_CUDA(dev_malloc(&h->d_btv, 6 * n * sizeof(double)));
  if (!h->d_btsc) HBX_CUDA(dev_malloc(&h->d_btsc, count * sizeof(hbx::MrScal)));
  if (!h->d_btdbl) HBX_CUDA(dev_malloc(&h->d_btdbl, 5 * (size_t)count * sizeof(double)));
  if (!h->d_btany) HBX_CUDA(dev_malloc(&h->d_btany, sizeof(int)));
  return HBX_OK;
}

}  // namespace

// The batched BiCGSTAB on h's instances, on stream s.  rtol (device,
// nullable): a tolerance per instance instead of tol.  true_res: also the
// true residual of every instance (one more product).  Per-instance results
// go to info (nullable, `count` entries); returns the first failing status.
static int batch_dev(hbx_hmat *h, const double *b, double *u, double tol, const double *rtol, int max_iter, int batch,
                     cudaStream_t s, bool true_res, hbx_solve_info *info) {
  const int count = h->inst_off.empty() ? 1 : (int)h->inst_off.size() - 1;
  int st = ensure_bt_workspace(h, count);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd;
  double *r = h->d_btv, *rh = r + n, *p = rh + n, *ap = p + n, *t = ap + n, *at = t + n;
  double *dots = h->d_btdbl, *bnorm = dots + 2 * (size_t)count, *tnorm = bnorm + count;
  HBX_CUDA(cudaEventRecord(h->ev0, s));
  // r = b - H u, rh = r, p = Ap = 0; the stop test of every instance
  HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, r), s));
  HBX_CUDA(hbx::bt_launch_setup(n, r, rh, p, ap, s));
  HBX_CUDA(hbx::bt_launch_dots(2, count, h->d_inst_off, r, r, b, b, dots, s));
  HBX_CUDA(hbx::bt_launch_init(count, dots, tol, rtol, max_iter, h->d_btsc, bnorm, h->d_btany, s));
  hbx::BtStep a{};
  a.n = n;
  a.count = count;
  a.max_iter = max_iter;
  a.off = h->d_inst_off;
  a.rinst = h->d_rinst;
  a.sc = h->d_btsc;
  a.any_active = h->d_btany;
  a.r = r; a.rh = rh; a.p = p; a.ap = ap; a.t = t; a.at = at; a.u = u; a.dots = dots; a.bnorm = bnorm;
  a.matvec = bt_matvec;
  a.ctx = h;
  // products inside the steps stream only the chunks of running instances
  const bool skip = h->d_chunk_inst && !skip_disabled();
  a.pre = skip ? h->d_inst_pre : nullptr;
  int any = 0, steps = 0, launches = 4;
  h->skip_inactive = skip ? 1 : 0;
  cudaError_t le = cudaSuccess;
  for (;;) {
    le = cudaMemcpyAsync(&any, h->d_btany, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess) le = cudaStreamSynchronize(s);
    if (le != cudaSuccess || !any || steps >= max_iter) break;
    for (int k = 0; k < batch && le == cudaSuccess; ++k) le = hbx::bt_launch_step(a, s);
    steps += batch;
    launches += (skip ? 13 : 11) * batch;
  }
  h->skip_inactive = 0;
  HBX_CUDA(le);
  HBX_CUDA(cudaEventRecord(h->ev1, s));
  if (true_res) {
    // the true residual of every instance: ||b - H u|| / ||b||
    HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, r), s));
    HBX_CUDA(hbx::bt_launch_dots(1, count, h->d_inst_off, r, r, nullptr, nullptr, tnorm, s));
    launches += 2;
  }
  std::vector<hbx::MrScal> sc(count);
  std::vector<double> hb(2 * (size_t)count);
  HBX_CUDA(cudaMemcpyAsync(sc.data(), h->d_btsc, count * sizeof(hbx::MrScal), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaMemcpyAsync(hb.data(), bnorm, 2 * (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  if ((st = check_device_error(h, s)) != HBX_OK) return st;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  int worst = HBX_OK;
  for (int k = 0; k < count; ++k) {
    const double bn = hb[k], tr = std::sqrt(hb[count + k]);
    const int stk = sc[k].status;
    if (stk != HBX_OK && worst == HBX_OK) worst = stk;
    if (info) {
      hbx_solve_info &I = info[k];
      std::memset(&I, 0, sizeof(I));
      I.iterations = sc[k].iters;
      I.status = stk;
      I.bnorm = bn;
      I.relres = bn > 0.0 ? std::sqrt(sc[k].rr) / bn : 0.0;
      I.true_relres = true_res ? (bn > 0.0 ? tr / bn : tr) : I.relres;
      I.seconds = ms * 1e-3;
      I.iter_launches = steps;
      I.launches = launches;
    }
  }
  return worst;
}

int hbx_bicgstab_batch(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info,
                       void *stream) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch: NULL argument");
  if (int rc = single_rhs(h, "hbx_bicgstab_batch")) return rc;
  const double tol = opts ? opts->tol : 1e-8;
  const int max_iter = opts ? opts->max_iter : 1000;
  const int batch = (opts && opts->batch > 0) ? opts->batch : 8;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch: bad tol or max_iter");
  const int st = batch_dev(h, b, u, tol, nullptr, max_iter, batch, static_cast<cudaStream_t>(stream), true, info);
  if (st != HBX_OK) return fail(st, std::string("hbx_bicgstab_batch: ") + hbx_status_string(st));
  return HBX_OK;
}

// Mixed-precision batched solve: the FP64 residual of every instance on h,
// the corrections by the batched BiCGSTAB on hl (FP32 or BF16 factors of the
// same instances), each instance's inner tolerance from its own residual;
// an instance leaves the outer loop once its FP64 residual meets tol.
static int batch_refined_dev(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                             hbx_solve_info *info, cudaStream_t s) {
  if (int rc = single_rhs(h, "hbx_bicgstab_batch_refined")) return rc;
  if (int rc = single_rhs(hl, "hbx_bicgstab_batch_refined")) return rc;
  const double tol = opts ? opts->tol : 1e-8;
  const int max_iter = opts ? opts->max_iter : 1000;
  const int batch = (opts && opts->batch > 0) ? opts->batch : 8;
  const double floor_tol = (opts && opts->inner_tol > 0.0) ? opts->inner_tol : 1e-6;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch_refined: bad tol or max_iter");
  const int count = h->inst_off.empty() ? 1 : (int)h->inst_off.size() - 1;
  int st = ensure_bt_workspace(h, count);
  if (st != HBX_OK) return st;
  const size_t n = (size_t)h->plan.nd;
  if (!hl->d_refine) HBX_CUDA(dev_malloc(&hl->d_refine, 2 * n * sizeof(double)));
  double *r = hl->d_refine, *d = hl->d_refine + n;
  // per-instance flags and inner tolerances (after the five per-instance
  // doubles of h's batch scalars, a free tail is not guaranteed: own buffer)
  if (!h->d_rflag) HBX_CUDA(dev_malloc(&h->d_rflag, (size_t)count * (sizeof(int) + sizeof(double)) + 16));
  int *d_flag = reinterpret_cast<int *>(h->d_rflag);
  double *d_itol = reinterpret_cast<double *>(reinterpret_cast<char *>(h->d_rflag) +
                                              ((size_t)count * sizeof(int) + 15) / 16 * 16);
  double *dots = h->d_btdbl;  // [count]: per-instance dots of the outer loop
  cudaEventRecord(h->ev2, s);
  std::vector<double> bb(count), rr(count), rel(count, 0.0), itol(count);
  std::vector<int> flag(count), inner(count, 0), status(count, HBX_ERR_NOT_CONVERGED), outer_k(count, 0);
  HBX_CUDA(hbx::bt_launch_dots(1, count, h->d_inst_off, b, b, nullptr, nullptr, dots, s));
  HBX_CUDA(cudaMemcpyAsync(bb.data(), dots, count * sizeof(double), cudaMemcpyDeviceToHost, s));
  HBX_CUDA(cudaStreamSynchronize(s));
  std::vector<hbx_solve_info> ii(count);
  int outer = 0, launches = 1;
  for (;;) {
    HBX_CUDA(mv_launch(h, matvec_args(h, -1.0, u, 1.0, b, r), s));
    HBX_CUDA(hbx::bt_launch_dots(1, count, h->d_inst_off, r, r, nullptr, nullptr, dots, s));
    HBX_CUDA(cudaMemcpyAsync(rr.data(), dots, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    HBX_CUDA(cudaStreamSynchronize(s));
    launches += 2;
    int active = 0;
    for (int k = 0; k < count; ++k) {
      const double bn = std::sqrt(bb[k]);
      rel[k] = bn > 0.0 ? std::sqrt(rr[k]) / bn : std::sqrt(rr[k]);
      flag[k] = 0;
      if (status[k] != HBX_ERR_NOT_CONVERGED) continue;  // finished or failed earlier
      if (!std::isfinite(rel[k])) status[k] = std::isfinite(bb[k]) ? HBX_ERR_BREAKDOWN : HBX_ERR_NONFINITE;
      else if (rel[k] < tol) status[k] = HBX_OK;
      else if (inner[k] < max_iter && outer < 64) {
        flag[k] = 1;
        itol[k] = std::max(floor_tol, 0.5 * tol / rel[k]);
        ++active;
      }
      outer_k[k] = outer;
    }
    if (!active) break;
    HBX_CUDA(cudaMemcpyAsync(d_flag, flag.data(), count * sizeof(int), cudaMemcpyHostToDevice, s));
    HBX_CUDA(cudaMemcpyAsync(d_itol, itol.data(), count * sizeof(double), cudaMemcpyHostToDevice, s));
    HBX_CUDA(hbx::bt_launch_mask(n, h->d_rinst, d_flag, r, s));
    HBX_CUDA(cudaMemsetAsync(d, 0, n * sizeof(double), s));
    int left = 0;
    for (int k = 0; k < count; ++k)
      if (flag[k]) left = std::max(left, max_iter - inner[k]);
    const int ist = batch_dev(hl, r, d, tol, d_itol, left, batch, s, false, ii.data());
    if (ist != HBX_OK && ist != HBX_ERR_NOT_CONVERGED && ist != HBX_ERR_BREAKDOWN) return fail(ist, "hbx_bicgstab_batch_refined: inner solve");
    for (int k = 0; k < count; ++k) {
      if (!flag[k]) continue;
      inner[k] += ii[k].iterations;
      if (ii[k].iterations == 0 && ii[k].status != HBX_OK) status[k] = ii[k].status;  // no progress possible
    }
    launches += ii[0].launches + 1;
    HBX_CUDA(hbx::launch_axpy(1.0, d, u, n, s));
    ++outer;
  }
  cudaEventRecord(h->ev3, s);
  HBX_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev2, h->ev3);
  int worst = HBX_OK;
  for (int k = 0; k < count; ++k) {
    if (status[k] != HBX_OK && worst == HBX_OK) worst = status[k];
    if (info) {
      hbx_solve_info &I = info[k];
      std::memset(&I, 0, sizeof(I));
      I.iterations = inner[k];
      I.outer = outer_k[k];
      I.status = status[k];
      I.bnorm = std::sqrt(bb[k]);
      I.relres = rel[k];
      I.true_relres = rel[k];
      I.seconds = ms * 1e-3;
      I.launches = launches;
    }
  }
  if ((st = check_device_error(h, s)) != HBX_OK) return st;
  if (worst != HBX_OK) return fail(worst, std::string("hbx_bicgstab_batch_refined: ") + hbx_status_string(worst));
  return HBX_OK;
}

int hbx_bicgstab_batch_refined(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                               hbx_solve_info *info, void *stream) {
  if (!h || !hl || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch_refined: NULL argument");
  if (h->plan.nd != hl->plan.nd || h->inst_off != hl->inst_off || h->device != hl->device)
    return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch_refined: h and hl must hold the same instances on one device");
  return batch_refined_dev(h, hl, b, u, opts, info, static_cast<cudaStream_t>(stream));
}

int hbx_bicgstab_batch_refined_host(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                                    hbx_solve_info *info) {
  if (!h || !hl || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch_refined_host: NULL argument");
  const size_t bytes = (size_t)h->plan.nd * sizeof(double);
  double *dv = nullptr;
  HBX_CUDA(dev_malloc(&dv, 2 * bytes));
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMemcpyAsync(dv, b, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dv + h->plan.nd, u, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) { cudaFree(dv); return cuda_fail(e, "hbx_bicgstab_batch_refined_host upload"); }
  int st = hbx_bicgstab_batch_refined(h, hl, dv, dv + h->plan.nd, opts, info, s);
  e = cudaMemcpyAsync(u, dv + h->plan.nd, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dv);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_bicgstab_batch_refined_host download");
  return st;
}

int hbx_bicgstab_batch_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts,
                            hbx_solve_info *info) {
  if (!h || !b || !u) return fail(HBX_ERR_INVALID, "hbx_bicgstab_batch_host: NULL argument");
  const size_t bytes = (size_t)h->plan.nd * sizeof(double);
  double *d = nullptr;
  HBX_CUDA(dev_malloc(&d, 2 * bytes));
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMemcpyAsync(d, b, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + h->plan.nd, u, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) { cudaFree(d); return cuda_fail(e, "hbx_bicgstab_batch_host upload"); }
  int st = hbx_bicgstab_batch(h, d, d + h->plan.nd, opts, info, s);
  e = cudaMemcpyAsync(u, d + h->plan.nd, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "hbx_bicgstab_batch_host download");
  return st;
}


void c_hacapk_adot_body_lfcpy_batch_sorted_(int *nd, stc_HACApK_leafmtxp *st_leafmtxp) {
  if (!nd || !st_leafmtxp) return;
  create_for(st_leafmtxp, *nd);
}

void c_hacapk_adot_body_lfmtx_batch_(double *zau, stc_HACApK_leafmtxp *st_leafmtxp, double *zu, double *zbu,
                                     double *time_batch, double *time_set, double *time_copy) {
  (void)zbu;
  (void)time_set;
  if (!st_leafmtxp || !zau || !zu) return;
  hbx_hmat *h = lookup(st_leafmtxp);
  if (!h) h = create_for(st_leafmtxp, st_leafmtxp->nd);
  if (!h) return;
  int rc = hbx_matvec_host(h, zu, zau, 1, time_batch, time_copy);
  if (rc != HBX_OK)
    std::fprintf(stderr, "!!!! hacapk_b200: matvec failed: %s (%s)\n", hbx_status_string(rc), hbx_last_error());
}

void c_hacapk_adot_body_lfdel_batch_(stc_HACApK_leafmtxp *st_leafmtxp) { release_for(st_leafmtxp); }

void c_hacapk_adot_body_lfcpy_gpu_(int *nd, stc_HACApK_leafmtxp *st_leafmtxp) {
  c_hacapk_adot_body_lfcpy_batch_sorted_(nd, st_leafmtxp);
}

void c_hacapk_adot_body_lfmtx_gpu_(double *zau, stc_HACApK_leafmtxp *st_leafmtxp, double *zu, double *zbu) {
  c_hacapk_adot_body_lfmtx_batch_(zau, st_leafmtxp, zu, zbu, nullptr, nullptr, nullptr);
}

void c_hacapk_adot_body_lfdel_gpu_(stc_HACApK_leafmtxp *st_leafmtxp) { release_for(st_leafmtxp); }

static int ctl_nrank(const stc_HACApK_lcontrol *ctl) {
  if (!ctl || !ctl->param) return 1;
  const int *lpmd = reinterpret_cast<const int *>(reinterpret_cast<const char *>(ctl->param) + ctl->lpmd_offset);
  return lpmd[1];
}

typedef int (*host_solver_fn)(hbx_hmat *, const double *, double *, const hbx_solve_opts *, hbx_solve_info *);

// The legacy device solvers: the engine of st_leafmtxp (made for the call
// when there is none), param(83) steps, param(91) tolerance, one rank.
static void legacy_device_solve(host_solver_fn solve, stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl,
                                double *u, double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  if (lrtrn) *lrtrn = HBX_OK;
  if (!st_leafmtxp || !u || !b || !param || !nd) {
    if (lrtrn) *lrtrn = HBX_ERR_INVALID;
    return;
  }
  if (ctl_nrank(st_ctl) > 1) {
    std::fprintf(stderr, "!!!! hacapk_b200: one MPI rank per solve only (nrank=%d)\n", ctl_nrank(st_ctl));
    if (lrtrn) *lrtrn = HBX_ERR_UNSUPPORTED;
    return;
  }
  hbx_hmat *h = lookup(st_leafmtxp);
  const bool own = (h == nullptr);
  if (own) h = create_for(st_leafmtxp, *nd);
  if (!h) {
    if (lrtrn) *lrtrn = HBX_ERR_CUDA;
    return;
  }
  hbx_solve_opts o{};
  o.tol = param[90];
  o.max_iter = (int)param[82];
  o.verbose = param[0] > 0 ? 1 : 0;
  o.restart = param[86] >= 1.0 && param[86] <= 64.0 ? (int)param[86] : 0;  // param(87): GCR's restart length
  hbx_solve_info info{};
  int rc = solve(h, b, u, &o, &info);
  if (nstp) *nstp = info.iterations;
  if (lrtrn) *lrtrn = rc;
  if (own) release_for(st_leafmtxp);
}

void c_hacapk_bicgstab_cax_lfmtx_gpu_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                      double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_bicgstab_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

// The two pipelined versions differ in where the reference overlaps its MPI
// gathers with the dot products; their arithmetic is the same, and so is the
// device sequence here (one GPU, no gathers).
void c_hacapk_bicgstab_cax_lfmtx_pipe_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                       double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_bicgstab_pipe_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

// GCR(m) with the solvers' argument list (the reference's GCR is the Fortran
// HACApK_gcrm_lfmtx, m_HACApK_solve.f90:506-571, chosen by param(85) = 2 in
// HACApK_solve, m_HACApK_use.f90:236-241; it has no C symbol): param(87) is
// the restart length, param(83) the step limit, param(91) the tolerance.
void c_hacapk_gcrm_lfmtx_gpu_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                              double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_gcr_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

void c_hacapk_bicgstab_cax_lfmtx_pipe2_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                        double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_bicgstab_pipe_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

// The reference's multi-GPU-per-process BiCGSTAB versions (HACApK_SOLVER.c:815
// mgpu1, :1405 mgpu2, :2137 mgpu3; its default build calls mgpu1 from
// HACApK_solve_cax, m_HACApK_use.f90:349).  They spread one process's leaves
// over gpus_per_proc GPUs (4 on that build), reduce the partial products by
// peer copies and run the _gpu_ recurrence with the vector operations
// repeated (1) or split (2, 3) over those GPUs.  Here a process drives one
// B200, which holds the whole H-matrix, so all three are the device BiCGSTAB
// on that GPU; several GPUs are one process each (the row-partitioned form).
// Like the reference's, they copy H in and release it after the solve unless
// an engine for st_leafmtxp already exists.
void c_hacapk_bicgstab_cax_lfmtx_mgpu1_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                        double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_bicgstab_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

void c_hacapk_bicgstab_cax_lfmtx_mgpu2_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                        double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_bicgstab_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

void c_hacapk_bicgstab_cax_lfmtx_mgpu3_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                        double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  legacy_device_solve(hbx_bicgstab_host, st_leafmtxp, st_ctl, u, b, param, nd, nstp, lrtrn);
}

// Host-vector BiCGSTAB with one GPU matvec per product (HACApK_SOLVER.c:254-417).
void c_hacapk_bicgstab_cax_lfmtx_flat_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl, double *u,
                                       double *b, double *param, int *nd, int *nstp, int *lrtrn) {
  if (lrtrn) *lrtrn = HBX_OK;
  if (!st_leafmtxp || !u || !b || !param || !nd || *nd <= 0) {
    if (lrtrn) *lrtrn = HBX_ERR_INVALID;
    return;
  }
  if (ctl_nrank(st_ctl) > 1) {
    if (lrtrn) *lrtrn = HBX_ERR_UNSUPPORTED;
    return;
  }
  hbx_hmat *h = lookup(st_leafmtxp);
  const bool own = (h == nullptr);
  if (own) h = create_for(st_leafmtxp, *nd);
  if (!h) {
    if (lrtrn) *lrtrn = HBX_ERR_CUDA;
    return;
  }
  for (int i = 0; i < *nd; ++i) {
    if (!std::isfinite(b[i]) || !std::isfinite(u[i])) {
      std::fprintf(stderr, "!!!! hacapk_b200: c_hacapk_bicgstab_cax_lfmtx_flat_: NaN or Inf in b or u (entry %d)\n", i);
      if (lrtrn) *lrtrn = HBX_ERR_NONFINITE;
      if (nstp) *nstp = 0;
      if (own) release_for(st_leafmtxp);
      return;
    }
  }
  int status = HBX_OK;
  auto gpu_mv = [](void *ctx, const double *x, double *y) -> int {
    return hbx_matvec_host(static_cast<hbx_hmat *>(ctx), x, y, 0, nullptr, nullptr);
  };
  const int steps = hbx::flat_bicgstab(*nd, u, b, param[90], (int)param[82], param[0] > 0 ? 1 : 0, gpu_mv, h,
                                       &status);
  if (lrtrn) *lrtrn = status;
  if (nstp) *nstp = steps;
  if (own) release_for(st_leafmtxp);
}

}  // extern "C"
