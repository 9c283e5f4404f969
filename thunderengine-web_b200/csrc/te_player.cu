// Tape player behind include/thunderstep.h: the reference's Replayer memory model
// (web/replay.js:46-121, 258-288) on one B200, CUDA kernels per dispatch, CUDA graphs
// for repeated steps, fused step phases in TE_MODE_FUSED (te_fused.cu).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/thunderstep.h"
#include "te_fused.cuh"
#include "te_json.hpp"
#include "te_kernels.cuh"
#include "te_player.hpp"

namespace te {

static constexpr uint64_t kAlign = 64;            // words per buffer alignment (replay.js:16)
static constexpr uint64_t kBytesSpare = 1u << 18;  // words for later step structures (replay.js:17)
static constexpr uint64_t kScratchCap = 1u << 26;  // words of per-thread scratch before y tiling (replay.js:18)

struct ApiError : std::runtime_error {
  int code;
  ApiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CU(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) throw ApiError(TE_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

cudaError_t opt_in_smem(const void* k, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;  // (kernel, device) -> bytes set
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[std::make_pair(k, dev)];
  if (have >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

// Step structure without setBytes data (replay.js:31): commands minus barriers, bytes
// replaced by their index and encoded length.
static std::string signature(const JValue& cmds) {
  std::string s;
  for (const JValue& c : cmds.arr) {
    const std::string& op = c.at("op").str;
    if (op == "barrier") {
      s += "|";
      continue;
    }
    if (op == "bytes") {
      s += "b" + std::to_string(c.at("index").i64()) + ":" + std::to_string(c.at("data").str.size()) + "|";
      continue;
    }
    s += op;
    for (auto& kv : c.obj) {
      if (kv.first == "op") continue;
      s += "," + kv.first + "=";
      if (kv.second.type == JValue::Str) s += kv.second.str;
      else if (kv.second.type == JValue::Arr) {
        for (auto& x : kv.second.arr) s += std::to_string(x.i64()) + ".";
      } else s += std::to_string((long long)kv.second.i64());
    }
    s += "|";
  }
  return s;
}

__global__ void k_region_hash(const uint32_t* __restrict__ M, uint64_t off, uint64_t len, uint32_t* H, uint32_t slot) {
  // Reference region hash (replay.js:407-418): sum over i of mix(M[off+i] ^ i*0x9E3779B1).
  uint32_t s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t ii = (uint32_t)i;
    uint32_t h = (M[off + i] ^ (ii * 0x9E3779B1u)) * 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    s += h;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&H[slot], s);
}

}  // namespace te

using namespace te;

namespace te {

// ------------------------------------------------------------------ planning

void Plan::load_kernel_meta(const char* kjson, size_t klen) {
  kmeta.clear();
  if (kjson && klen) {
    JValue root = JParser(kjson, klen).parse();
    for (auto& kv : root.obj) {
      KMeta m;
      m.scratch = (uint64_t)(kv.second.get("scratch") ? kv.second.at("scratch").i64() : 0);
      for (auto& p : kv.second.at("params").arr)
        m.params.push_back({(int)p.at("index").i64(), p.at("kind").str == "ref", p.at("write").truthy()});
      kmeta[kv.first] = m;
    }
  } else {
    int n;
    const KernelSpec* t = kernel_table(&n);
    for (int i = 0; i < n; i++) {
      KMeta m;
      for (int q = 0; q < t[i].nparams; q++)
        m.params.push_back({t[i].params[q].index, t[i].params[q].kind != kPtr, t[i].params[q].write != 0});
      kmeta[t[i].name] = m;
    }
  }
}

std::map<int, uint64_t> Plan::layout_bytes(const JValue& cmds) {
  // setBytes payloads (replay.js:68-83): each at bytesTop, advanced by 4-word blocks + 4
  std::map<int, uint64_t> offs;
  for (size_t i = 0; i < cmds.arr.size(); i++) {
    const JValue& c = cmds.arr[i];
    if (c.at("op").str != "bytes") continue;
    std::vector<uint8_t> raw = base64_decode(c.at("data").str);
    uint64_t words = ceil_div(raw.size(), 4);
    if (bytes_spare_end && bytes_top + words + 4 > bytes_spare_end)
      throw ApiError(TE_ERANGE, "no room for the bytes of a new step structure (BYTES_SPARE)");
    offs[(int)i] = bytes_top;
    raw.resize(words * 4, 0);
    bytes_init.emplace_back(bytes_top, raw);
    bytes_top += ceil_div(words, 4) * 4 + 4;
  }
  return offs;
}

uint64_t Plan::region_len(uint64_t off) const {
  // regionLen (replay.js:168-178): arena field or rest of the buffer
  for (int b = (int)buffers.size() - 1; b >= 0; b--) {
    if (off >= base[b]) {
      uint64_t end = base[b] + buffers[b].length / 4;
      if (buffers[b].arena) return std::min<uint64_t>(field_stride / 4, end - off);
      return end - off;
    }
  }
  return 0;
}

std::vector<Op> Plan::build_ops(const JValue& cmds, const std::map<int, uint64_t>& offs, bool hashes) {
  // buildOps (replay.js:85-121)
  std::vector<Op> ops;
  std::map<int, uint64_t> bind;
  std::map<int, int64_t> last;
  std::string pipe;
  for (size_t i = 0; i < cmds.arr.size(); i++) {
    const JValue& c = cmds.arr[i];
    const std::string& op = c.at("op").str;
    if (op == "pipe") {
      pipe = c.at("name").str;
    } else if (op == "buf") {
      int idx = (int)c.at("index").i64();
      int64_t b = c.at("buf").i64();
      if (b >= (int64_t)buffers.size()) throw ApiError(TE_EINVAL, "buffer id out of range");
      bind[idx] = b < 0 ? 0 : base[b] + (uint64_t)c.at("offset").i64() / 4;
      last[idx] = b;
    } else if (op == "bufoff") {
      int idx = (int)c.at("index").i64();
      auto it = last.find(idx);
      if (it == last.end() || it->second < 0) throw ApiError(TE_EINVAL, "bufoff without a buffer");
      bind[idx] = base[it->second] + (uint64_t)c.at("offset").i64() / 4;
    } else if (op == "bytes") {
      bind[(int)c.at("index").i64()] = offs.at((int)i);
    } else if (op == "end") {
      bind.clear();
    } else if (op == "copy") {
      Op o;
      o.copy = true;
      o.name = "copy";
      o.src = base[c.at("src").i64()] + (uint64_t)c.at("srcOffset").i64() / 4;
      o.dst = base[c.at("dst").i64()] + (uint64_t)c.at("dstOffset").i64() / 4;
      o.n = (uint64_t)c.at("size").i64() / 4;
      ops.push_back(o);
    } else if (op == "dispatch") {
      auto km = kmeta.find(pipe);
      if (km == kmeta.end()) throw ApiError(TE_ENOKERNEL, "no kernel " + pipe);
      const KernelSpec* spec = find_kernel(pipe.c_str());
      if (!spec && !(flags & TE_FLAG_DEFER_MISSING)) throw ApiError(TE_ENOKERNEL, "no CUDA kernel for " + pipe);
      if (c.get("kind") && c.at("kind").str != "threads")
        throw ApiError(TE_EINVAL, "dispatch kind " + c.at("kind").str + " not supported");
      Op o;
      o.copy = false;
      o.spec = spec;
      o.name = pipe;
      for (int d = 0; d < 3; d++) {
        o.grid[d] = (int)c.at("grid").arr.at(d).i64();
        o.tg[d] = (int)c.at("tg").arr.at(d).i64();
      }
      uint64_t threads = (uint64_t)o.grid[0] * o.grid[1] * o.grid[2];
      uint64_t tileY = o.grid[1];
      if (km->second.scratch && km->second.scratch * threads > kScratchCap) {
        uint64_t row = km->second.scratch * o.grid[0] * o.grid[2];
        tileY = std::max<uint64_t>(o.tg[1], (kScratchCap / row / o.tg[1]) * o.tg[1]);
      }
      scratch_need = std::max<uint64_t>(scratch_need, km->second.scratch * o.grid[0] * o.grid[2] * tileY);
      o.tile_y = tileY;
      o.bind = bind;
      if (hashes) {
        for (auto& p : km->second.params) {
          if (!p.write) continue;
          HashReq h;
          h.slot = hash_count++;
          auto it = bind.find(p.index);
          h.bound = it != bind.end();
          h.off = h.bound ? it->second : 0;
          h.len = h.bound ? region_len(h.off) : 0;
          o.hashes.push_back(h);
        }
      }
      ops.push_back(o);
    }
  }
  return ops;
}

void Plan::plan(const char* tj, size_t tl, bool with_hashes_) {
  JValue tape = JParser(tj, tl).parse();
  buffers.clear();
  for (auto& b : tape.at("buffers").arr) buffers.push_back({(uint64_t)b.at("length").i64(), b.get("arena") && b.at("arena").truthy()});
  field_stride = (uint64_t)tape.at("fieldStride").i64();
  uint64_t top = 0;
  base.clear();
  for (auto& b : buffers) {
    base.push_back(top);
    top += ceil_div(ceil_div(b.length, 4), kAlign) * kAlign;
  }
  buffers_end = top;
  bytes_top = top;
  bytes_spare_end = 0;
  scratch_need = 0;
  hash_count = 0;
  with_hashes = with_hashes_;
  bytes_init.clear();
  const JValue& s0 = tape.at("steps").arr.at(0);
  static const JValue empty_arr = [] { JValue v; v.type = JValue::Arr; return v; }();
  const JValue* diag = tape.get("diag");
  if (!diag || diag->type != JValue::Arr) diag = &empty_arr;
  auto e0 = layout_bytes(s0);
  auto eD = layout_bytes(*diag);
  bytes_spare_end = bytes_top + kBytesSpare;
  top = ceil_div(bytes_spare_end, kAlign) * kAlign;
  cache.clear();
  Step st;
  st.ops = build_ops(s0, e0, with_hashes);
  st.offs = e0;
  for (size_t i = 0; i < s0.arr.size(); i++)
    if (s0.arr[i].at("op").str == "bytes") st.data[(int)i] = s0.arr[i].at("data").str;
  std::string sig = signature(s0);
  cache[sig] = std::move(st);
  active = &cache[sig];
  diag_ops = build_ops(*diag, eD, false);
  scratch_base = top;
  top += ceil_div(scratch_need, kAlign) * kAlign;
  mem_words = top;
  host_bytes.assign(bytes_spare_end - buffers_end, 0);
  for (auto& bi : bytes_init) std::memcpy(&host_bytes[bi.first - buffers_end], bi.second.data(), bi.second.size());
}

void Plan::finalize_args(std::vector<Op>& ops) {
  for (Op& o : ops) {
    if (o.copy || !o.spec) continue;
    KArgs& A = o.args;
    std::memset(&A, 0, sizeof(A));
    A.bx = o.tile[0];
    A.by = o.tile[1];
    A.gx = o.grid[0];
    A.gy = o.grid[1];
    A.gz = o.grid[2];
    auto word = [&](uint64_t off) -> uint32_t {
      if (off < buffers_end || off >= bytes_spare_end)
        throw ApiError(TE_EINVAL, o.name + ": parameter struct bound outside the setBytes area");
      uint32_t w;
      std::memcpy(&w, &host_bytes[off - buffers_end], 4);
      return w;
    };
    auto fl = [&](uint64_t off) {
      uint32_t w = word(off);
      float f;
      std::memcpy(&f, &w, 4);
      return f;
    };
    auto it0 = o.bind.find(0);
    if (it0 == o.bind.end()) throw ApiError(TE_EINVAL, o.name + ": GridDims (binding 0) not bound");
    uint64_t gd = it0->second;
    A.ref0 = M + gd;
    A.scr = reinterpret_cast<float*>(M + scratch_base);
    A.scr_rows = (unsigned)std::min<uint64_t>(o.tile_y, 0xffffffffu);
    A.g.nx = (int)word(gd + 0);
    A.g.ny = (int)word(gd + 1);
    A.g.nz = (int)word(gd + 2);
    A.g.sJ = (int)word(gd + 3);
    A.g.sK = (int)word(gd + 4);
    A.g.rdx = fl(gd + 5);
    A.g.rdy = fl(gd + 6);
    A.g.rdz = fl(gd + 7);
    // host-side bounds check of the grid every kernel indexes with (int32 field indices)
    {
      const Dims& g = A.g;
      bool ok = g.nx >= 1 && g.ny >= 1 && g.nz >= 1 && g.nx < (1 << 20) && g.ny < (1 << 20) && g.nz < (1 << 20) &&
                g.sJ >= g.nx + 7 && g.sK >= g.ny + 7;
      uint64_t count = ok ? (uint64_t)g.sJ * g.sK * (g.nz + 1) : 0;
      ok = ok && count < (1ull << 31) && (field_stride == 0 || count * 4 <= field_stride);
      if (!ok) throw ApiError(TE_EINVAL, o.name + ": GridDims out of range or larger than the arena field stride");
    }
    if (o.spec->acoustic) {
      auto it1 = o.bind.find(1);
      if (it1 == o.bind.end()) throw ApiError(TE_EINVAL, o.name + ": AcousticParams (binding 1) not bound");
      uint64_t ap = it1->second;
      A.a.dts = fl(ap + 0);
      A.a.alph = fl(ap + 1);
      A.a.beta = fl(ap + 2);
      A.a.kdiv = fl(ap + 3);
      A.a.smeps = fl(ap + 4);
    }
    int nvec = 0;
    for (int q = 0; q < o.spec->nparams; q++) {
      const ParamSpec& ps = o.spec->params[q];
      auto it = o.bind.find(ps.index);
      if (ps.kind == kPtr) {
        if (it != o.bind.end()) {
          if (it->second >= buffers_end) throw ApiError(TE_ERANGE, o.name + ": pointer binding outside the tape buffers");
          A.p[ps.index] = reinterpret_cast<float*>(M + it->second);
        }
      } else if (ps.index >= 1 && !(ps.index == 1 && o.spec->acoustic)) {
        if (it == o.bind.end()) continue;
        if (ps.kind == kRef && it->second < buffers_end) {
          // a parameter struct that lives in a tape buffer (the radar head of
          // morr_refl10cm): the kernel reads its words through the pointer
          A.p[ps.index] = reinterpret_cast<float*>(M + it->second);
          continue;
        }
        A.iv[ps.index] = (int)word(it->second);
        A.f[ps.index] = fl(it->second);
        A.iv2[ps.index] = (int)word(it->second + 1);
        if (ps.kind == kRefS) {
          if (nvec == 2) throw ApiError(TE_EINVAL, o.name + ": more than two struct parameters read by words");
          for (int w = 0; w < 8; w++)  // words past the end of the setBytes area read 0
            A.sw[nvec][w] = it->second + w < bytes_spare_end ? fl(it->second + w) : 0.0f;
          nvec++;
        }
      }
    }
    // morr_column keeps 29 per-column arrays of nz levels in the scratch the reference sizes
    // for 128 levels (3712 words per thread), one thread per column
    if (o.name == "morr_column" && (A.g.nz < 1 || A.g.nz > 128 || o.grid[2] != 1 || !o.tile_y))
      throw ApiError(TE_EINVAL, o.name + ": needs 1 <= nz <= 128 and a one-level dispatch grid");
    // morr_refl10cm: 11 per-column arrays of nz levels in its 1408 scratch words, and reads
    // the 14-word radar head, 100 bins of 6 words for snow and for graupel and 100 weights
    // from tape buffers
    if (o.name == "morr_refl10cm") {
      if (A.g.nz < 1 || A.g.nz > 128 || o.grid[2] != 1 || !o.tile_y)
        throw ApiError(TE_EINVAL, o.name + ": needs 1 <= nz <= 128 and a one-level dispatch grid");
      const uint64_t need[5] = {0, 14, 600, 600, 100};
      for (int b = 1; b <= 13; b++) {
        if (!A.p[b]) throw ApiError(TE_EINVAL, o.name + ": binding " + std::to_string(b) + " not bound");
        if (b <= 4 && o.bind.at(b) + need[b] > buffers_end)
          throw ApiError(TE_ERANGE, o.name + ": binding " + std::to_string(b) + " runs past the tape buffers");
      }
    }
    // turb_zero writes up to level nz + 1 of its binding (its own range check): the
    // highest word the dispatch grid reaches must lie in the planned memory
    if (o.name == "turb_zero" && A.p[1]) {
      const uint64_t gi = std::min<uint64_t>(o.grid[0], A.g.sJ), gj = std::min<uint64_t>(o.grid[1], A.g.sK);
      const uint64_t gk = std::min<uint64_t>(o.grid[2], (uint64_t)A.g.nz + 2);
      const uint64_t top = o.bind.at(1) + (gi - 1) + (uint64_t)A.g.sJ * ((gj - 1) + (uint64_t)A.g.sK * (gk - 1));
      if (gi && gj && gk && top >= mem_words) throw ApiError(TE_ERANGE, o.name + ": dispatch writes past the planned memory");
    }
    // the __restrict__ build is valid when no written region overlaps another bound region
    bool disjoint = true;
    for (int q1 = 0; q1 < o.spec->nparams && disjoint; q1++) {
      const ParamSpec& a = o.spec->params[q1];
      auto ia = o.bind.find(a.index);
      if (a.kind != kPtr || ia == o.bind.end()) continue;
      const uint64_t a0 = ia->second, a1 = a0 + region_len(a0);
      for (int q2 = q1 + 1; q2 < o.spec->nparams && disjoint; q2++) {
        const ParamSpec& b = o.spec->params[q2];
        auto ib = o.bind.find(b.index);
        if (b.kind != kPtr || ib == o.bind.end() || !(a.write || b.write)) continue;
        const uint64_t b0 = ib->second, b1 = b0 + region_len(b0);
        if (a0 < b1 && b0 < a1) disjoint = false;
      }
    }
    const KernelSpec* f = disjoint ? fast::find_kernel(o.spec->name) : nullptr;
    o.launch = f ? f->launch : o.spec->launch;
  }
}

}  // namespace te

// ------------------------------------------------------------------ C ABI

static int fail(te_ctx* ctx, int code, const std::string& m) {
  if (ctx) ctx->err = m;
  return code;
}

#define API_BEGIN(ctx) \
  if (!ctx) return TE_EINVAL; \
  try {
#define API_END(ctx)                                              \
  }                                                               \
  catch (const te::ApiError& e) { return fail(ctx, e.code, e.what()); } \
  catch (const std::exception& e) { return fail(ctx, TE_EINVAL, e.what()); } \
  return TE_OK;

static void require_plan(te_ctx* ctx) {
  if (!ctx->plan.M) throw te::ApiError(TE_ESTATE, "te_plan has not been called");
}

extern "C" {

int te_create(const te_config* cfg, te_ctx** out) {
  if (!out) return TE_EINVAL;
  *out = nullptr;
  te_ctx* ctx = new te_ctx();
  ctx->device = cfg ? cfg->device : 0;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    ctx->err = std::string("cuda init: ") + cudaGetErrorString(e);
    *out = ctx;
    return TE_ECUDA;
  }
  ctx->plan.stream = ctx->stream;
  ctx->plan.flags = cfg ? cfg->flags : 0;
  *out = ctx;
  return TE_OK;
}

int te_plan(te_ctx* ctx, const char* tape_json, size_t tape_len, const char* kernels_json, size_t kernels_len,
            int with_hashes) {
  API_BEGIN(ctx)
  if (!tape_json) throw te::ApiError(TE_EINVAL, "no tape");
  CU(cudaSetDevice(ctx->device));
  te::Plan& P = ctx->plan;
  P.release();
  P.load_kernel_meta(kernels_json, kernels_len);
  P.plan(tape_json, tape_len, with_hashes != 0);
  CU(cudaMalloc(&P.M, P.mem_words * 4));
  CU(cudaMemsetAsync(P.M, 0, P.mem_words * 4, ctx->plan.stream));
  CU(cudaMalloc(&P.H, std::max<size_t>(16, (size_t)P.hash_count * 4)));
  CU(cudaMemsetAsync(P.H, 0, std::max<size_t>(16, (size_t)P.hash_count * 4), ctx->plan.stream));
  for (auto& bi : P.bytes_init)
    CU(cudaMemcpyAsync(P.M + bi.first, bi.second.data(), bi.second.size(), cudaMemcpyHostToDevice, ctx->plan.stream));
  CU(cudaStreamSynchronize(ctx->plan.stream));
  P.bytes_init.clear();
  P.finalize_args(P.active->ops);
  P.finalize_args(P.diag_ops);
  P.fused_dirty = true;
  API_END(ctx)
}

int te_get_info(te_ctx* ctx, te_info* out) {
  API_BEGIN(ctx)
  require_plan(ctx);
  const te::Plan& P = ctx->plan;
  out->mem_words = P.mem_words;
  out->buffers_end = P.buffers_end;
  out->scratch_base = P.scratch_base;
  out->hash_count = P.hash_count;
  out->num_buffers = (uint32_t)P.buffers.size();
  out->num_ops = (uint32_t)P.active->ops.size();
  uint32_t nd = 0;
  for (auto& o : P.active->ops) nd += o.copy ? 0 : 1;
  out->num_dispatches = nd;
  API_END(ctx)
}

int te_buffer_base(te_ctx* ctx, int buf_id, uint64_t* word_off) {
  API_BEGIN(ctx)
  require_plan(ctx);
  if (buf_id < 0 || buf_id >= (int)ctx->plan.buffers.size()) throw te::ApiError(TE_EINVAL, "buffer id out of range");
  *word_off = ctx->plan.base[buf_id];
  API_END(ctx)
}

int te_write_words(te_ctx* ctx, uint64_t word_off, const void* data, size_t bytes) {
  API_BEGIN(ctx)
  require_plan(ctx);
  te::Plan& P = ctx->plan;
  if (word_off + te::ceil_div(bytes, 4) > P.mem_words) throw te::ApiError(TE_ERANGE, "write past the end of memory");
  CU(cudaSetDevice(ctx->device));
  CU(cudaMemcpyAsync(P.M + word_off, data, bytes, cudaMemcpyHostToDevice, ctx->plan.stream));
  CU(cudaStreamSynchronize(ctx->plan.stream));
  // keep the host copy of the parameter area in step with device memory
  uint64_t lo = std::max<uint64_t>(word_off, P.buffers_end), hi = std::min<uint64_t>(word_off + bytes / 4, P.bytes_spare_end);
  if (lo < hi) {
    std::memcpy(&P.host_bytes[lo - P.buffers_end], (const uint8_t*)data + (lo - word_off) * 4, (hi - lo) * 4);
    P.finalize_args(P.active->ops);
    P.finalize_args(P.diag_ops);
    P.invalidate_graphs();
  }
  API_END(ctx)
}

int te_write_words_async(te_ctx* ctx, uint64_t word_off, const void* data, size_t bytes) {
  API_BEGIN(ctx)
  require_plan(ctx);
  te::Plan& P = ctx->plan;
  if (word_off + te::ceil_div(bytes, 4) > P.buffers_end)
    throw te::ApiError(TE_ERANGE, "asynchronous writes must stay inside the tape buffers");
  CU(cudaSetDevice(ctx->device));
  CU(cudaMemcpyAsync(P.M + word_off, data, bytes, cudaMemcpyHostToDevice, ctx->plan.stream));
  API_END(ctx)
}

int te_read_async(te_ctx* ctx, uint64_t word_off, uint64_t words, void* out) {
  API_BEGIN(ctx)
  require_plan(ctx);
  if (word_off + words > ctx->plan.mem_words) throw te::ApiError(TE_ERANGE, "read past the end of memory");
  CU(cudaSetDevice(ctx->device));
  CU(cudaMemcpyAsync(out, ctx->plan.M + word_off, words * 4, cudaMemcpyDeviceToHost, ctx->plan.stream));
  API_END(ctx)
}

int te_upload(te_ctx* ctx, int buf_id, const void* data, size_t bytes) {
  if (!ctx) return TE_EINVAL;
  if (!ctx->plan.M) return fail(ctx, TE_ESTATE, "te_plan has not been called");
  if (buf_id < 0 || buf_id >= (int)ctx->plan.buffers.size()) return fail(ctx, TE_EINVAL, "buffer id out of range");
  if (bytes > ctx->plan.buffers[buf_id].length + 3) return fail(ctx, TE_ERANGE, "upload larger than the buffer");
  return te_write_words(ctx, ctx->plan.base[buf_id], data, bytes);
}

int te_use_step(te_ctx* ctx, const char* cmds_json, size_t len) {
  API_BEGIN(ctx)
  require_plan(ctx);
  te::Plan& P = ctx->plan;
  te::JValue cmds = te::JParser(cmds_json, len).parse();
  if (cmds.type != te::JValue::Arr) throw te::ApiError(TE_EINVAL, "step must be a JSON array of commands");
  std::string sig = te::signature(cmds);
  auto it = P.cache.find(sig);
  if (it == P.cache.end()) {
    te::Step st;
    st.offs = P.layout_bytes(cmds);
    st.ops = P.build_ops(cmds, st.offs, false);
    uint64_t need = P.scratch_base + te::ceil_div(P.scratch_need, te::kAlign) * te::kAlign;
    if (need > P.mem_words) throw te::ApiError(TE_ERANGE, "new step structure needs more kernel scratch than planned");
    for (auto& bi : P.bytes_init) {
      std::memcpy(&P.host_bytes[bi.first - P.buffers_end], bi.second.data(), bi.second.size());
      CU(cudaMemcpyAsync(P.M + bi.first, bi.second.data(), bi.second.size(), cudaMemcpyHostToDevice, ctx->plan.stream));
    }
    P.bytes_init.clear();
    it = P.cache.emplace(sig, std::move(st)).first;
  }
  te::Step& e = it->second;
  bool changed = (&e != P.active);
  for (size_t i = 0; i < cmds.arr.size(); i++) {
    const te::JValue& c = cmds.arr[i];
    if (c.at("op").str != "bytes") continue;
    auto d = e.data.find((int)i);
    if (d != e.data.end() && d->second == c.at("data").str) continue;
    e.data[(int)i] = c.at("data").str;
    std::vector<uint8_t> raw = te::base64_decode(c.at("data").str);
    raw.resize(te::ceil_div(raw.size(), 4) * 4, 0);
    uint64_t off = e.offs.at((int)i);
    std::memcpy(&P.host_bytes[off - P.buffers_end], raw.data(), raw.size());
    CU(cudaMemcpyAsync(P.M + off, raw.data(), raw.size(), cudaMemcpyHostToDevice, ctx->plan.stream));
    changed = true;
  }
  CU(cudaStreamSynchronize(ctx->plan.stream));
  P.active = &e;
  if (changed) {
    P.finalize_args(P.active->ops);
    P.invalidate_graphs();
  }
  API_END(ctx)
}

int te_run_ops(te_ctx* ctx, int first_op, int last_op, int with_hashes) {
  API_BEGIN(ctx)
  require_plan(ctx);
  CU(cudaSetDevice(ctx->device));
  te::Plan& P = ctx->plan;
  int n = (int)P.active->ops.size();
  if (first_op < 0) first_op = 0;
  if (last_op >= n) last_op = n - 1;
  P.launch_exact(P.active->ops, first_op, last_op, with_hashes != 0);
  CU(cudaGetLastError());
  API_END(ctx)
}

int te_run(te_ctx* ctx, int nsteps, int with_hashes) {
  API_BEGIN(ctx)
  require_plan(ctx);
  CU(cudaSetDevice(ctx->device));
  te::Plan& P = ctx->plan;
  for (int s = 0; s < nsteps; s++) {
    if (with_hashes) P.launch_exact(P.active->ops, 0, (int)P.active->ops.size() - 1, true);
    else P.launch_step_graph();
  }
  CU(cudaGetLastError());
  API_END(ctx)
}

int te_run_diag(te_ctx* ctx) {
  API_BEGIN(ctx)
  require_plan(ctx);
  CU(cudaSetDevice(ctx->device));
  ctx->plan.launch_exact(ctx->plan.diag_ops, 0, (int)ctx->plan.diag_ops.size() - 1, false);
  CU(cudaGetLastError());
  API_END(ctx)
}

int te_read(te_ctx* ctx, uint64_t word_off, uint64_t words, void* out) {
  API_BEGIN(ctx)
  require_plan(ctx);
  if (word_off + words > ctx->plan.mem_words) throw te::ApiError(TE_ERANGE, "read past the end of memory");
  CU(cudaSetDevice(ctx->device));
  CU(cudaMemcpyAsync(out, ctx->plan.M + word_off, words * 4, cudaMemcpyDeviceToHost, ctx->plan.stream));
  CU(cudaStreamSynchronize(ctx->plan.stream));
  API_END(ctx)
}

int te_read_hashes(te_ctx* ctx, uint32_t* out, size_t n) {
  API_BEGIN(ctx)
  require_plan(ctx);
  size_t m = std::min<size_t>(n, ctx->plan.hash_count);
  CU(cudaSetDevice(ctx->device));
  if (m) CU(cudaMemcpyAsync(out, ctx->plan.H, m * 4, cudaMemcpyDeviceToHost, ctx->plan.stream));
  CU(cudaStreamSynchronize(ctx->plan.stream));
  API_END(ctx)
}

int te_clear_hashes(te_ctx* ctx) {
  API_BEGIN(ctx)
  require_plan(ctx);
  CU(cudaSetDevice(ctx->device));
  CU(cudaMemsetAsync(ctx->plan.H, 0, std::max<size_t>(16, (size_t)ctx->plan.hash_count * 4), ctx->plan.stream));
  API_END(ctx)
}

int te_device_ptr(te_ctx* ctx, uint64_t word_off, void** out) {
  API_BEGIN(ctx)
  require_plan(ctx);
  if (word_off >= ctx->plan.mem_words) throw te::ApiError(TE_ERANGE, "offset outside memory");
  *out = ctx->plan.M + word_off;
  API_END(ctx)
}

int te_set_mode(te_ctx* ctx, int mode) {
  API_BEGIN(ctx)
  if (mode != TE_MODE_EXACT && mode != TE_MODE_FUSED) throw te::ApiError(TE_EINVAL, "unknown mode");
  ctx->plan.mode = mode;
  ctx->plan.invalidate_graphs();
  API_END(ctx)
}

int te_fused_segments(te_ctx* ctx, te_segment* out, int max, int* count) {
  API_BEGIN(ctx)
  require_plan(ctx);
  te::Plan& P = ctx->plan;
  if (P.fused_dirty || P.fused.segs.empty()) {
    P.fused.build(P, P.active->ops);
    P.fused_dirty = false;
  }
  int n = (int)P.fused.segs.size();
  if (count) *count = n;
  for (int i = 0; i < n && i < max && out; i++) {
    const te::FusedSegment& s = P.fused.segs[i];
    out[i].kind = s.kind;
    out[i].first_op = s.first;
    out[i].last_op = s.last;
    out[i].kernels = s.kind == 0 ? 0 : (s.kind == 1 ? 3 : 1);
    if (s.kind == 0)
      for (int q = s.first; q <= s.last; q++) out[i].kernels += P.active->ops[q].copy ? 0 : 1;
  }
  API_END(ctx)
}

int te_run_segment(te_ctx* ctx, int seg, int part) {
  API_BEGIN(ctx)
  require_plan(ctx);
  CU(cudaSetDevice(ctx->device));
  te::Plan& P = ctx->plan;
  if (P.fused_dirty || P.fused.segs.empty()) {
    P.fused.build(P, P.active->ops);
    P.fused_dirty = false;
  }
  if (seg < 0 || seg >= (int)P.fused.segs.size()) throw te::ApiError(TE_EINVAL, "segment out of range");
  P.fused.launch_segment(P, P.active->ops, seg, part);
  CU(cudaGetLastError());
  API_END(ctx)
}

const char* te_op_name(te_ctx* ctx, int op) {
  if (!ctx || !ctx->plan.active || op < 0 || op >= (int)ctx->plan.active->ops.size()) return nullptr;
  return ctx->plan.active->ops[op].name.c_str();
}

int te_set_stream(te_ctx* ctx, void* cuda_stream) {
  API_BEGIN(ctx)
  CU(cudaSetDevice(ctx->device));
  CU(cudaStreamSynchronize(ctx->plan.stream));
  ctx->plan.stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->stream;
  ctx->plan.invalidate_graphs();
  API_END(ctx)
}

size_t te_kernel_table_json(char* buf, size_t n) {
  int cnt;
  const te::KernelSpec* t = te::kernel_table(&cnt);
  std::string s = "{";
  for (int i = 0; i < cnt; i++) {
    if (i) s += ",";
    s += "\"" + std::string(t[i].name) + "\":{\"params\":[";
    for (int q = 0; q < t[i].nparams; q++) {
      if (q) s += ",";
      s += "{\"index\":" + std::to_string(t[i].params[q].index) + ",\"kind\":\"" +
           (t[i].params[q].kind != te::kPtr ? "ref" : "ptr") + "\",\"write\":" + (t[i].params[q].write ? "true" : "false") + "}";
    }
    s += "]}";
  }
  s += "}";
  if (buf && n) {
    size_t m = std::min(n - 1, s.size());
    std::memcpy(buf, s.data(), m);
    buf[m] = 0;
  }
  return s.size();
}

int te_sync(te_ctx* ctx) {
  API_BEGIN(ctx)
  CU(cudaSetDevice(ctx->device));
  CU(cudaStreamSynchronize(ctx->plan.stream));
  API_END(ctx)
}

void te_destroy(te_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->plan.release();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* te_last_error(te_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

uint32_t te_region_hash_host(const uint32_t* w, uint64_t n) {
  uint32_t s = 0;
  for (uint64_t i = 0; i < n; i++) {
    uint32_t h = (w[i] ^ ((uint32_t)i * 0x9E3779B1u)) * 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    s += h;
  }
  return s;
}

}  // extern "C"

// ------------------------------------------------------------ execution

namespace te {

void Plan::launch_exact(std::vector<Op>& ops, int first, int last, bool hashes) {
  for (int i = first; i <= last; i++) {
    Op& o = ops[i];
    if (o.copy) {
      CU(cudaMemcpyAsync(M + o.dst, M + o.src, o.n * 4, cudaMemcpyDeviceToDevice, stream));
      continue;
    }
    if (!o.spec) throw ApiError(TE_ENOKERNEL, "no CUDA kernel for " + o.name);
    (o.launch ? o.launch : o.spec->launch)(o.args, stream);
    if (hashes) {
      for (auto& h : o.hashes) {
        if (!h.bound || !h.len) continue;
        launch_kernel(k_region_hash, dim3(64), dim3(256), 0, stream, M, h.off, h.len, H, h.slot);
      }
    }
  }
}

void Plan::invalidate_graphs() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  graph_exec = nullptr;
  fused_dirty = true;
}

cudaGraph_t Plan::capture_step() {
  if (mode == TE_MODE_FUSED && fused_dirty) {
    fused.build(*this, active->ops);
    fused_dirty = false;
  }
  cudaGraph_t graph = nullptr;
  CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  try {
    if (mode == TE_MODE_FUSED) fused.launch(*this, active->ops);
    else launch_exact(active->ops, 0, (int)active->ops.size() - 1, false);
  } catch (...) {
    cudaStreamEndCapture(stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  CU(cudaStreamEndCapture(stream, &graph));
  return graph;
}

void Plan::launch_step_graph() {
  if (!graph_exec) {
    cudaGraph_t graph = capture_step();
    cudaError_t e = cudaGraphInstantiate(&graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    CU(e);
  }
  CU(cudaGraphLaunch(graph_exec, stream));
}

void Plan::release() {
  release_adjoint(*this);
  invalidate_graphs();
  fused.release();
  if (M) cudaFree(M);
  if (H) cudaFree(H);
  M = nullptr;
  H = nullptr;
  cache.clear();
  active = nullptr;
  diag_ops.clear();
}

}  // namespace te
