// context.cuh -- the fmmb200_ctx object: stream, grow-only device buffers,
// error state and the device-resident state of the last forward.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

struct fmmb200_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // the host-pointer forward copies the momenta here while the stream starts the tree
  // build on the positions; ev_copy[0]: positions copied, [1]: momenta copied
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copy[2] = {};
  std::string err;
  int64_t fail_alloc_countdown = 0;  // >0: the countdown-th next allocation fails
  bool timing = false;
  cudaEvent_t ev[16] = {};
  bool ev_ready = false;

  struct Buf {
    void *p = nullptr;
    size_t cap = 0;
  };
  std::map<std::string, Buf> bufs;  // named device buffers, grow-only (caching)
  size_t device_bytes = 0;

  // pinned host scratch for small readbacks (counts, histograms, flags)
  void *h_pinned = nullptr;
  size_t h_pinned_cap = 0;
  int *d_status = nullptr;  // device status word (DeviceStatus)

  // ---- state of the last tree / forward ----
  bool have_tree = false;    // tree arrays valid
  bool have_lists = false;   // interaction lists valid
  bool have_forward = false; // expansions of a forward valid
  bool saved = false;        // forward saved for backward
  bool pavg_from_momenta = true;  // p_avg = sum(u)/N was computed here (so it depends on u)
  int64_t N = 0, N0 = 0;
  int n = 0, precision = 0;
  int ml = 0;
  int64_t nc = 0, nleaf = 0, leaf0 = 0, max_leaf = 0;
  int64_t nm2l = 0, np2p = 0;
  double eta = 0.0, charge = 0.0, lambda = 1.0;
  double pavg[3] = {0, 0, 0}, stretch[3] = {1, 1, 1};
  int traversal_steps = 0;
  int list_bits = 1;  // pair keys are (target << list_bits) | source
  int m2l_engine = 0;  // FMMB200_M2L_*: mixed-form M2L engine
  bool tree_reuse = false;  // forward: refit the previous tree when it is still exact
  // forward: fields of the leaves [rank nleaf / world, (rank + 1) nleaf / world) only
  int shard_rank = 0, shard_world = 1;
  // traversal target filter of a memory-sharded rank: only the rows of the level-trav_L
  // cluster trav_g, its descendants and its ancestors (trav_L < 0: every row)
  int trav_L = -1, trav_g = 0;
  // largest pair counts and frontier a traversal of this context has needed (the next
  // traversal sizes its buffers from them)
  int64_t trav_need_p = 0, trav_need_m = 0, trav_need_f = 0;
  double trav_key[4] = {-1, -1, -1, -1};  // (clusters, eta, filter level, filter cluster) of those needs
  // the M2L target lists the M2L launchers read (a shard's compacted copy, or all)
  const char *m2l_ptr_key = "m2l_ptr";
  const char *m2l_src_key = "m2l_src";
  fmmb200_stats stats{};

  // pairwise-summation plan for p_avg (depends on N only)
  int64_t pw_N = -1;
  int pw_nleaf = 0, pw_nint = 0, pw_root = 0;
  std::vector<int> pw_hoff;  // internal nodes grouped by height

  int fail(int code, const std::string &msg) {
    err = msg;
    return code;
  }

  // Device buffer `name` with at least `bytes` bytes (contents not preserved on growth).
  // Buffer `name` of at least `bytes`, reallocated (contents lost) only when smaller.  A new
  // allocation gets 1/8 headroom, so `bytes` must be a need: a request derived from another
  // buffer's capacity would grow by that headroom on every call.
  int ensure_bytes(const char *name, size_t bytes, void **out) {
    Buf &b = bufs[name];
    if (bytes == 0) bytes = 16;
    if (b.cap < bytes) {
      if (b.p) {
        cudaStreamSynchronize(stream);  // the old buffer may still be read by queued work
        cudaFree(b.p);
        device_bytes -= b.cap;
        b.p = nullptr;
        b.cap = 0;
      }
      if (fail_alloc_countdown > 0 && --fail_alloc_countdown == 0) {
        return fail(FMMB200_ERR_OUT_OF_MEMORY,
                    std::string("injected allocation failure for buffer '") + name + "'");
      }
      size_t want = bytes + bytes / 8;  // headroom so that small growth does not reallocate
      want = (want + 255) & ~(size_t)255;
      cudaError_t e = cudaMalloc(&b.p, want);
      if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return fail(FMMB200_ERR_OUT_OF_MEMORY, std::string("cudaMalloc(") + std::to_string(want) +
                                                   " B) for '" + name + "': " + cudaGetErrorString(e));
      }
      b.cap = want;
      device_bytes += want;
    }
    *out = b.p;
    return FMMB200_OK;
  }

  template <class T>
  int ensure(const char *name, int64_t count, T **out) {
    void *p = nullptr;
    int s = ensure_bytes(name, (size_t)(count > 0 ? count : 1) * sizeof(T), &p);
    *out = (T *)p;
    return s;
  }

  template <class T>
  T *get(const char *name) {
    auto it = bufs.find(name);
    return it == bufs.end() ? nullptr : (T *)it->second.p;
  }

  int pinned(size_t bytes, void **out) {
    if (h_pinned_cap < bytes) {
      if (h_pinned) cudaFreeHost(h_pinned);
      h_pinned = nullptr;
      h_pinned_cap = 0;
      cudaError_t e = cudaMallocHost(&h_pinned, bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FMMB200_ERR_OUT_OF_MEMORY, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
      }
      h_pinned_cap = bytes;
    }
    *out = h_pinned;
    return FMMB200_OK;
  }

  int sync() {
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(FMMB200_ERR_CUDA, std::string("stream sync: ") + cudaGetErrorString(e));
    return FMMB200_OK;
  }

  int64_t launches = 0;  // kernels launched by this context (counted at each check)

  int check_launch(const char *what, int nlaunched = 1) {
    launches += nlaunched;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FMMB200_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return FMMB200_OK;
  }

  // Reads and clears the device status word (synchronises the stream).
  int check_device_status(const char *what) {
    int *h = nullptr;
    FMM_TRY(pinned(sizeof(int) * 4, (void **)&h));
    cudaError_t e = cudaMemcpyAsync(h, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(FMMB200_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    int st = h[0];
    if (st != fmmb200::kDevOk) {
      cudaMemsetAsync(d_status, 0, sizeof(int), stream);
      return fail(FMMB200_ERR_DEVICE, std::string(what) + ": device status " + std::to_string(st) +
                                          (st == fmmb200::kDevQueueOverflow ? " (bounded wait expired)" : " (index check)"));
    }
    return FMMB200_OK;
  }
};

using Ctx = fmmb200_ctx;
