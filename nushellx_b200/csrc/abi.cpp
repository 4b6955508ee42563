// extern "C" entry points of libnsx (declared in include/nsx.h).  Every call
// catches internal failures and turns them into a negative return code plus a
// thread-local message: nothing is thrown or aborted across the boundary.
#include <atomic>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>
#include <exception>
#include <new>
#include <map>
#include "nsx_internal.h"

namespace nsx {
static thread_local std::string g_err;
void fail(int code, const std::string &msg) { throw Error{code, msg}; }
void check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  int code = (e == cudaErrorMemoryAllocation) ? NSX_E_NOMEM : NSX_E_CUDA;
  throw Error{code, std::string(what) + ": " + cudaGetErrorString(e)};
}
void solve(nsx_handle *h, const nsx_params *P, const nsx_state *resume, nsx_state *state_out, double *evals,
           double *evecs, nsx_report *rep);
std::shared_ptr<void> load_files(const nsx_files *f, nsx_problem *p);
std::shared_ptr<void> compress_problem(const nsx_problem *p, const nsx_dop *d, nsx_problem *out);
std::shared_ptr<DopArrays> read_dop(const std::string &path);
int noalloc_guarded(nsx_handle *h, const double *x, double *y, void *stream);

// Device calls on a handle: a plan-only handle (created with device < 0) has no device data.
static void require_device(const nsx_handle *h) {
  if (h->device < 0) fail(NSX_E_ARG, "the handle was created without a device (plan only)");
}
// Calls that need whole products (solves, expectation values): a shard needs its exchange.
void require_full_product(const nsx_handle *h) {
  if (h->shard_world > 1 && !h->exch)
    fail(NSX_E_ARG, "the handle is one of " + std::to_string(h->shard_world) +
                        " output-block shards: set an exchange (nsx_set_exchange) before solving");
}

template <typename F>
static int guarded(F &&f) {
  try {
    f();
    return NSX_OK;
  } catch (const Error &e) {
    g_err = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    g_err = "host allocation failed";
    return NSX_E_NOMEM;
  } catch (const std::exception &e) {
    g_err = e.what();
    return NSX_E_ARG;
  } catch (...) {
    g_err = "unknown failure";
    return NSX_E_ARG;
  }
}
}  // namespace nsx

using namespace nsx;

extern "C" {

const char *nsx_last_error(void) { return g_err.c_str(); }

// A handle for rank `rank` of `world` output-block shards (world = 1: the whole product).
static int create_handle(const nsx_problem *prob, int device, int rank, int world, nsx_handle **out) {
  if (!out) {
    g_err = "null output handle pointer";
    return NSX_E_ARG;
  }
  *out = nullptr;
  nsx_handle *h = new (std::nothrow) nsx_handle();
  if (!h) {
    g_err = "host allocation failed";
    return NSX_E_NOMEM;
  }
  int rc = guarded([&] {
    if (!prob) fail(NSX_E_ARG, "null problem");
    if (world < 1 || world > 1024) fail(NSX_E_ARG, "world size out of range (1 .. 1024)");
    if (rank < 0 || rank >= world) fail(NSX_E_ARG, "rank out of range (0 .. world - 1)");
    h->device = device < 0 ? -1 : device;
    build_plan(h, prob);   // every block: the flops of each block's rows
    if (world == 1) {
      h->shard_first = {0, (int)h->blocks.size()};
    } else {
      h->shard_first = split_blocks(h->block_flops, world);
      h->shard_rank = rank;
      h->shard_world = world;
      h->own_b0 = h->shard_first[rank];
      h->own_b1 = h->shard_first[rank + 1];
      build_plan(h, prob);   // this rank's blocks only
    }
    if (device < 0) return;   // plan only: no CUDA call at all
    DeviceGuard dg(device);
    upload(h);
  });
  if (rc != NSX_OK) {
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return NSX_OK;
}

int nsx_create(const nsx_problem *prob, int device, nsx_handle **out) {
  return create_handle(prob, device, 0, 1, out);
}

int nsx_create_shard(const nsx_problem *prob, int device, int32_t rank, int32_t world, nsx_handle **out) {
  return create_handle(prob, device, rank, world, out);
}

int nsx_load_files_shard(const nsx_files *files, int device, int32_t rank, int32_t world, nsx_handle **out) {
  nsx_problem p;
  std::memset(&p, 0, sizeof(p));
  std::shared_ptr<void> store;
  int rc = guarded([&] {
    if (!files || !out) fail(NSX_E_ARG, "null argument");
    store = load_files(files, &p);
  });
  if (rc != NSX_OK) return rc;
  return create_handle(&p, device, rank, world, out);
}

int nsx_load_files(const nsx_files *files, int device, nsx_handle **out) {
  return nsx_load_files_shard(files, device, 0, 1, out);
}

int nsx_shard_info(const nsx_handle *h, int32_t *rank, int32_t *world, int64_t *row_begin, double *est_flops) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    if (rank) *rank = h->shard_rank;
    if (world) *world = h->shard_world;
    const int nbl = (int)h->blocks.size();
    for (int r = 0; r <= h->shard_world; ++r) {
      const int b = h->shard_first[r];
      if (row_begin) row_begin[r] = b < nbl ? h->blocks[b].off : h->no_state;
      if (est_flops && r < h->shard_world) {
        double f = 0.0;
        for (int k = b; k < h->shard_first[r + 1]; ++k) f += h->block_flops[k];
        est_flops[r] = f;
      }
    }
  });
}

int nsx_block_flops(const nsx_handle *h, double *out) {
  return guarded([&] {
    if (!h || !out) fail(NSX_E_ARG, "null argument");
    for (size_t i = 0; i < h->block_flops.size(); ++i) out[i] = h->block_flops[i];
  });
}

int nsx_set_exchange(nsx_handle *h, nsx_exchange_fn fn, void *user) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    h->exch = fn;
    h->exch_user = user;
  });
}

int nsx_create_z(const nsx_problem *prob, const nsx_dop *dop, int device, nsx_handle **out) {
  nsx_problem z;
  std::memset(&z, 0, sizeof(z));
  std::shared_ptr<void> store;
  int rc = guarded([&] {
    if (!prob || !dop || !out) fail(NSX_E_ARG, "null argument");
    store = compress_problem(prob, dop, &z);
  });
  if (rc != NSX_OK) return rc;
  return nsx_create(&z, device, out);
}

int nsx_load_files_z(const nsx_files *files, const char *dop_path, int device, nsx_handle **out) {
  nsx_problem p, z;
  std::memset(&p, 0, sizeof(p));
  std::memset(&z, 0, sizeof(z));
  std::shared_ptr<void> store, zstore;
  int rc = guarded([&] {
    if (!files || !dop_path || !out) fail(NSX_E_ARG, "null argument");
    store = load_files(files, &p);
    auto dop = read_dop(dop_path);
    nsx_dop d = dop->view();
    zstore = compress_problem(&p, &d, &z);
  });
  if (rc != NSX_OK) return rc;
  return nsx_create(&z, device, out);
}

int nsx_set_interaction(nsx_handle *h, const double *op_vals, int32_t nop, const double *a_seg_vals, int64_t a_nvals,
                        const double *b_seg_vals, int64_t b_nvals) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    set_interaction(h, op_vals, nop, a_seg_vals, a_nvals, b_seg_vals, b_nvals);
    DeviceGuard dg(h->device);
    if (h->device >= 0) upload_interaction(h, a_seg_vals, b_seg_vals);
  });
}

int nsx_batch_solve(nsx_handle *const *handles, int32_t n, const nsx_params *params, double *const *evals,
                    double *const *evecs, nsx_report *reports) {
  int rc = guarded([&] {
    if (!handles || !params || !evals) fail(NSX_E_ARG, "null argument");
    if (n < 0 || n > 4096) fail(NSX_E_ARG, "problem count out of range (0 .. 4096)");
    std::vector<nsx_handle *> hs(handles, handles + n);
    for (int i = 0; i < n; ++i) {
      if (!hs[i] || !evals[i]) fail(NSX_E_ARG, "null handle or eigenvalue array for problem " + std::to_string(i));
      if (hs[i]->device < 0) fail(NSX_E_ARG, "problem " + std::to_string(i) + ": the handle was created without a device (plan only)");
      require_full_product(hs[i]);
      for (int j = 0; j < i; ++j)
        if (hs[j] == hs[i]) fail(NSX_E_ARG, "the same handle is listed twice (problems " + std::to_string(j) +
                                                " and " + std::to_string(i) + ")");
    }
  });
  if (rc != NSX_OK || n == 0) return rc;
  // one host worker per handle at a time, each solving on its handle's own stream
  std::vector<int> codes(n, NSX_OK);
  std::vector<std::string> msgs(n);
  std::atomic<int> next{0};
  const int workers = std::min<int>(n, 32);
  std::vector<std::thread> pool;
  for (int w = 0; w < workers; ++w)
    pool.emplace_back([&] {
      for (int i = next++; i < n; i = next++) {
        codes[i] = guarded([&] {
          NSX_CUDA(cudaSetDevice(handles[i]->device));
          solve(handles[i], &params[i], nullptr, nullptr, evals[i], evecs ? evecs[i] : nullptr,
                reports ? &reports[i] : nullptr);
        });
        if (codes[i] != NSX_OK) msgs[i] = g_err;
      }
    });
  for (auto &t : pool) t.join();
  for (int i = 0; i < n; ++i)
    if (codes[i] != NSX_OK) {
      g_err = "problem " + std::to_string(i) + ": " + msgs[i];
      return codes[i];
    }
  return NSX_OK;
}

int nsx_write_results(const nsx_handle *h, const char *prefix, const double *evals, const double *evecs,
                      int32_t nev, int32_t iterations, const char *intfile, int32_t T2) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    write_results(h, prefix, evals, evecs, nev, iterations, intfile, T2);
  });
}

int nsx_write_state(const nsx_handle *h, const char *prefix, const nsx_state *state, const double *evals,
                    const double *evecs, int32_t nev, const char *intfile, int32_t T2) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    write_state(h, prefix, state, evals, evecs, nev, intfile, T2);
  });
}

int nsx_read_state(const nsx_handle *h, const char *prefix, nsx_state *state) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    read_state(h, prefix, state);
  });
}

int64_t nsx_dim(const nsx_handle *h) { return h ? h->no_state : 0; }
int32_t nsx_nblocks(const nsx_handle *h) { return h ? (int32_t)h->blocks.size() : 0; }

int nsx_blocks(const nsx_handle *h, int32_t *blocks4, int64_t *offsets) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    for (size_t i = 0; i < h->blocks.size(); ++i) {
      if (blocks4) {
        blocks4[4 * i + 0] = h->blocks[i].J2a;
        blocks4[4 * i + 1] = h->blocks[i].J2b;
        blocks4[4 * i + 2] = h->blocks[i].da;
        blocks4[4 * i + 3] = h->blocks[i].db;
      }
      if (offsets) offsets[i] = h->blocks[i].off;
    }
    if (offsets) offsets[h->blocks.size()] = h->no_state;
  });
}

int nsx_lcoef(const nsx_handle *h, uint8_t *mask) {
  return guarded([&] {
    if (!h || !mask) fail(NSX_E_ARG, "null argument");
    std::memcpy(mask, h->lcoef.data(), h->lcoef.size());
  });
}

double nsx_matvec_flops(const nsx_handle *h) {
  return h ? h->flops_like + h->flops_y + h->flops_mix + h->flops_a : 0.0;
}

int nsx_matvec(nsx_handle *h, const double *x, double *y, int32_t precision, void *stream) {
  return guarded([&] {
    if (!h || !x || !y) fail(NSX_E_ARG, "null argument");
    if (x == y) fail(NSX_E_ARG, "x and y must not alias");
    require_device(h);
    DeviceGuard dg(h->device);
    matvec_device(h, x, y, precision, (cudaStream_t)stream);
  });
}

int nsx_matvec_noalloc(nsx_handle *h, const double *x, double *y, void *stream) {
  return guarded([&] { noalloc_guarded(h, x, y, stream); });
}

int nsx_matvec_host(nsx_handle *h, const double *x, double *y, int32_t precision) {
  return guarded([&] {
    if (!h || !x || !y) fail(NSX_E_ARG, "null argument");
    require_device(h);
    DeviceGuard dg(h->device);
    size_t bytes = sizeof(double) * h->no_state;
    NSX_CUDA(cudaMemcpy(h->d.xin, x, bytes, cudaMemcpyHostToDevice));
    matvec_device(h, h->d.xin, h->d.xout, precision, 0);
    if (h->shard_world > 1 && !h->exch) {   // this rank's rows only; the others stay as they were
      NSX_CUDA(cudaMemcpy(y + h->row0, h->d.xout + h->row0, sizeof(double) * (h->row1 - h->row0),
                          cudaMemcpyDeviceToHost));
    } else {
      NSX_CUDA(cudaMemcpy(y, h->d.xout, bytes, cudaMemcpyDeviceToHost));
    }
    check_device_error(h);
  });
}

int nsx_expectation_matrix(nsx_handle *h, const double *vecs, int32_t nvec, int32_t precision, double *out) {
  return guarded([&] {
    if (!h || !vecs || !out) fail(NSX_E_ARG, "null argument");
    require_device(h);
    require_full_product(h);
    DeviceGuard dg(h->device);
    expectation_matrix(h, vecs, nvec, precision, out);
    check_device_error(h);
  });
}

int nsx_xpct_files(nsx_handle *h, const char *xvc_path, const char *out_prefix, int32_t precision) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    require_device(h);
    require_full_product(h);
    DeviceGuard dg(h->device);
    xpct_files(h, xvc_path, out_prefix, precision);
    check_device_error(h);
  });
}

int nsx_solve(nsx_handle *h, const nsx_params *params, double *evals, double *evecs, nsx_report *report) {
  return guarded([&] {
    if (!h || !params || !evals) fail(NSX_E_ARG, "null argument");
    require_device(h);
    require_full_product(h);
    DeviceGuard dg(h->device);
    solve(h, params, nullptr, nullptr, evals, evecs, report);
    check_device_error(h);
  });
}

int nsx_solve_ex(nsx_handle *h, const nsx_params *params, const nsx_state *resume, nsx_state *state_out,
                 double *evals, double *evecs, nsx_report *report) {
  return guarded([&] {
    if (!h || !params || !evals) fail(NSX_E_ARG, "null argument");
    require_device(h);
    require_full_product(h);
    DeviceGuard dg(h->device);
    solve(h, params, resume, state_out, evals, evecs, report);
    check_device_error(h);
  });
}

int nsx_stats_reset(nsx_handle *h, int32_t timing) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    DeviceGuard dg(h->device);
    flush_stage_events(h);
    h->launches = h->matvecs = 0;
    for (int i = 0; i < NSX_STAGES; ++i) {
      h->stage_launches[i] = 0;
      h->stage_ms[i] = 0;
    }
    h->timing = timing != 0;
  });
}

int nsx_get_stats(nsx_handle *h, nsx_stats *out) {
  return guarded([&] {
    if (!h || !out) fail(NSX_E_ARG, "null argument");
    DeviceGuard dg(h->device);
    flush_stage_events(h);
    if (h->device >= 0) check_device_error(h);
    out->launches = h->launches;
    out->matvecs = h->matvecs;
    // algorithmic figures for the precision of the last H.v
    int prec = h->last_precision;
    stage_bytes_flops(h, prec, out->stage_bytes, out->stage_flops);
    for (int i = 0; i < NSX_STAGES; ++i) {
      out->stage_launches[i] = h->stage_launches[i];
      out->stage_ms[i] = h->stage_ms[i];
    }
  });
}

int nsx_get_plan_info(const nsx_handle *h, nsx_plan_info *out) {
  return guarded([&] {
    if (!h || !out) fail(NSX_E_ARG, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->y_elems = h->y_elems;
    out->zbar_elems = h->z_elems;
    out->zbar_tc_elems = h->z32_elems;
    for (const auto &g : h->ygroups)
      out->y_row_tiles_max = std::max(out->y_row_tiles_max, (g.m + KY_TILE_ROWS - 1) / KY_TILE_ROWS);
    out->group_sources_max = h->max_zns;
    out->fused_fp32 = h->max_zns <= 16 ? 1 : 0;   // KYZ_NS
    std::map<std::pair<int64_t, int32_t>, int> pieces;   // (slab out offset, col0) -> K pieces
    for (const auto &t : h->atiles) {
      out->slab_rows_max = std::max(out->slab_rows_max, t.k_end);
      out->slab_nl_max = std::max(out->slab_nl_max, t.nl);
      out->slab_splits_max = std::max(out->slab_splits_max, ++pieces[{t.out, t.col0}]);
    }
    for (int c = 0; c < 4; ++c) out->tc_tiles[c] = h->atc_off[c + 1] - h->atc_off[c];
    for (const auto &t : h->atiles_tc) out->tc_chunks_max = std::max<int64_t>(out->tc_chunks_max, (t.kgroups + 3) / 4);
    out->fp32_path = h->fp32_path;
    for (const auto &t : h->atiles_tc) out->tc_pieces += t.split;
  });
}

int nsx_set_fp32_path(nsx_handle *h, int32_t path) {
  return guarded([&] {
    if (!h) fail(NSX_E_ARG, "null handle");
    set_fp32_path(h, path);
  });
}

void nsx_destroy(nsx_handle *h) {
  if (!h) return;
  try {
    DeviceGuard dg(h->device);
    release(h);
  } catch (...) {
    release(h);   // the device could not be made current: free what the current context can
  }
  delete h;
}

}  // extern "C"
