// C-ABI entry points (include/vulcan_b200.h): network set-up and the
// stream-ordered launch sequences of the Ros2 step and the block solver.
#include <cuda_runtime.h>

#include <cstdio>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "vb_common.cuh"
#include "vb_launch.cuh"


struct VbNet {
  vb::NetDev dev;
  void* base;
  size_t bytes;
  VbTuning tune;
};

static thread_local std::string g_err;

// ---- optional per-launch event profiling (see vb_profile in the header)
namespace {
struct ProfSite {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
};
bool g_prof = false;
ProfSite g_sites[VB_PROFILE_SITES];

struct ProfScope {
  int site;
  cudaStream_t st;
  cudaEvent_t b = nullptr, e = nullptr;
  ProfScope(int s, cudaStream_t stream) : site(s), st(stream) {
    if (g_prof) {
      cudaEventCreate(&b);
      cudaEventCreate(&e);
      cudaEventRecord(b, st);
    }
  }
  ~ProfScope() {
    if (g_prof && b) {
      cudaEventRecord(e, st);
      g_sites[site].ev.emplace_back(b, e);
    }
  }
};
}  // namespace

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

static int cuda_fail(cudaError_t e, const char* where) {
  return fail(VB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define VB_CHECK(call, where)                      \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return cuda_fail(_e, where); \
  } while (0)

// ---- scratch of vb_ros2_step_static
// One copy of this array lives on every device that loads the library, for
// the life of the process. Host code may not use `g_step_scratch` as an
// address: the device address is looked up once per device with that device
// current (cudaGetSymbolAddress) and cached.
static __device__ __align__(256) double g_step_scratch[VB_STATIC_SCRATCH_BYTES / sizeof(double)];

namespace {
constexpr int kScratchDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kScratchDevices] = {};
}  // namespace

static int static_scratch(double** out) {
  int dev = 0;
  VB_CHECK(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kScratchDevices) return fail(VB_ERR_ARG, "device ordinal beyond the static scratch table");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    VB_CHECK(cudaGetSymbolAddress(&p, g_step_scratch), "cudaGetSymbolAddress(static scratch)");
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return VB_OK;
}

extern "C" {

const char* vb_last_error(void) { return g_err.c_str(); }
int vb_version(void) { return 1; }

int vb_net_create(int ni, int nr, int T, const int64_t* r_idx, const int64_t* p_idx, const double* r_st,
                  const double* p_st, const uint8_t* three, VbNet** out) {
  if (!out || !r_idx || !p_idx || !r_st || !p_st || !three) return fail(VB_ERR_ARG, "null argument");
  if (ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "ni must be in [1, 128]");
  if (nr < 1 || T < 1 || T > 8) return fail(VB_ERR_ARG, "nr >= 1 and 1 <= max_terms <= 8 required");
  const int R = nr + 1;
  for (int64_t e = 0; e < (int64_t)R * T; ++e) {
    if (r_idx[e] < 0 || r_idx[e] > ni || p_idx[e] < 0 || p_idx[e] > ni)
      return fail(VB_ERR_ARG, "species index out of [0, ni]");
  }
  // gather tables in segment_sum order (increasing flat index)
  std::vector<std::vector<int32_t>> loss(ni), prod(ni), jac((size_t)ni * ni);
  for (int rs = 0; rs < R * T; ++rs) {
    if (r_idx[rs] < ni) loss[r_idx[rs]].push_back(rs);
    if (p_idx[rs] < ni) prod[p_idx[rs]].push_back(rs);
  }
  for (int r = 0; r < R; ++r)
    for (int o = 0; o < 2 * T; ++o) {
      int64_t row = o < T ? r_idx[(int64_t)r * T + o] : p_idx[(int64_t)r * T + (o - T)];
      for (int s = 0; s < T; ++s) {
        int64_t col = r_idx[(int64_t)r * T + s];
        if (row < ni && col < ni) jac[row * ni + col].push_back((int32_t)(((int64_t)r * 2 * T + o) * T + s));
      }
    }
  auto csr = [](const std::vector<std::vector<int32_t>>& lists, std::vector<int32_t>& ptr,
                std::vector<int32_t>& ent) {
    ptr.assign(lists.size() + 1, 0);
    for (size_t i = 0; i < lists.size(); ++i) ptr[i + 1] = ptr[i] + (int32_t)lists[i].size();
    ent.clear();
    for (auto& l : lists) ent.insert(ent.end(), l.begin(), l.end());
    if (ent.empty()) ent.push_back(0);
  };
  std::vector<int32_t> lp, le, pp, pe, jp, je;
  csr(loss, lp, le);
  csr(prod, pp, pe);
  csr(jac, jp, je);
  // packed term words and the table of distinct coefficients
  if ((int64_t)R * T > 0xffff) return fail(VB_ERR_ARG, "(nr+1)*max_terms must stay below 65536");
  std::vector<double> coefs;
  std::map<uint64_t, int> coef_id;
  bool too_many = false;
  auto cid_of = [&](double c) {
    uint64_t bits;
    std::memcpy(&bits, &c, sizeof bits);
    auto it = coef_id.find(bits);
    if (it != coef_id.end()) return it->second;
    if ((int)coefs.size() >= vb::MAX_COEF) { too_many = true; return 0; }
    int id = (int)coefs.size();
    coefs.push_back(c);
    coef_id[bits] = id;
    return id;
  };
  std::vector<uint32_t> lw(le.size()), pw(pe.size()), jw(je.size());
  for (size_t e = 0; e < le.size(); ++e) lw[e] = vb::term_word(le[e] / T, cid_of(r_st[le[e]]));
  for (size_t e = 0; e < pe.size(); ++e) pw[e] = vb::term_word(pe[e] / T, cid_of(p_st[pe[e]]));
  for (size_t e = 0; e < je.size(); ++e) {
    int fe = je[e], s = fe % T, ro = fe / T, o = ro % (2 * T), r = ro / (2 * T);
    double c = o < T ? -r_st[(int64_t)r * T + o] : p_st[(int64_t)r * T + (o - T)];
    jw[e] = vb::term_word(r * T + s, cid_of(c));
  }
  if (too_many) return fail(VB_ERR_ARG, "more than 256 distinct stoichiometric coefficients");
  if (coefs.empty()) coefs.push_back(0.0);
  // destinations in decreasing term count (ties: increasing index); threads
  // take them in rank bands (thread t: ranks t, t + LAYER_THREADS, ...) so the
  // lanes of a warp sum lists of similar length. The term words of each group
  // of 32 consecutive ranks are interleaved: term i of rank q at
  // base(q / 32) + 32 i + q % 32, the group padded to its longest list (the
  // first rank's), so a warp holding a group loads one line per term.
  // Descriptor of rank q: its first word, then count | row << 16 | col << 24
  // (one load per destination).
  std::vector<uint32_t> order(2 * (size_t)ni * ni), jwi;
  {
    const size_t nd = (size_t)ni * ni;
    std::vector<int32_t> perm(nd);
    for (size_t d = 0; d < nd; ++d) perm[d] = (int32_t)d;
    std::stable_sort(perm.begin(), perm.end(),
                     [&](int32_t x, int32_t y) { return jp[x + 1] - jp[x] > jp[y + 1] - jp[y]; });
    std::vector<size_t> gbase((nd + 31) / 32 + 1, 0);
    for (size_t g = 0; g + 1 < gbase.size(); ++g) {
      const int32_t d = perm[32 * g];
      gbase[g + 1] = gbase[g] + 32 * (size_t)(jp[d + 1] - jp[d]);
    }
    if (gbase.back() > 0xffffffffu) return fail(VB_ERR_ARG, "Jacobian gather table too large");
    jwi.assign(std::max<size_t>(gbase.back(), 1), 0u);
    for (size_t q = 0; q < nd; ++q) {
      const uint32_t d = (uint32_t)perm[q];
      const uint32_t cnt = (uint32_t)(jp[d + 1] - jp[d]);
      if (cnt > 0xffffu) return fail(VB_ERR_ARG, "a Jacobian entry has more than 65535 terms");
      const size_t first = gbase[q / 32] + q % 32;
      for (uint32_t i = 0; i < cnt; ++i) jwi[first + 32 * (size_t)i] = jw[jp[d] + i];
      order[2 * q] = (uint32_t)first;
      order[2 * q + 1] = cnt | ((d / (uint32_t)ni) << 16) | ((d % (uint32_t)ni) << 24);
    }
  }
  // species lists t = 2 i (loss), 2 i + 1 (production), words interleaved by
  // groups of 32 consecutive lists (term k of list t at base(t / 32) + 32 k +
  // t % 32, each group padded to its longest list); descriptor {first, count}
  std::vector<uint32_t> sdesc(4 * (size_t)ni), swi;
  {
    const size_t nl = 2 * (size_t)ni;
    auto len = [&](size_t t) -> size_t {
      const std::vector<int32_t>& ptr = (t & 1) ? pp : lp;
      return (size_t)(ptr[t / 2 + 1] - ptr[t / 2]);
    };
    std::vector<size_t> gbase((nl + 31) / 32 + 1, 0);
    for (size_t g = 0; g + 1 < gbase.size(); ++g) {
      size_t mx = 0;
      for (size_t t = 32 * g; t < std::min(nl, 32 * g + 32); ++t) mx = std::max(mx, len(t));
      gbase[g + 1] = gbase[g] + 32 * mx;
    }
    if (gbase.back() > 0xffffffffu) return fail(VB_ERR_ARG, "species gather table too large");
    swi.assign(std::max<size_t>(gbase.back(), 1), 0u);
    for (size_t t = 0; t < nl; ++t) {
      const std::vector<int32_t>& ptr = (t & 1) ? pp : lp;
      const std::vector<uint32_t>& w = (t & 1) ? pw : lw;
      const size_t first = gbase[t / 32] + t % 32, n = len(t);
      for (size_t k = 0; k < n; ++k) swi[first + 32 * k] = w[ptr[t / 2] + k];
      sdesc[2 * t] = (uint32_t)first;
      sdesc[2 * t + 1] = (uint32_t)n;
    }
  }
  // species lists in natural order (t = 2 i loss, 2 i + 1 production)
  std::vector<int32_t> snp(2 * (size_t)ni + 1, 0);
  std::vector<uint32_t> snw;
  for (int t = 0; t < 2 * ni; ++t) {
    const std::vector<int32_t>& ptr = (t & 1) ? pp : lp;
    const std::vector<uint32_t>& w = (t & 1) ? pw : lw;
    for (int32_t e = ptr[t / 2]; e < ptr[t / 2 + 1]; ++e) snw.push_back(w[e]);
    snp[t + 1] = (int32_t)snw.size();
  }
  if (snw.empty()) snw.push_back(0u);
  std::vector<int32_t> ri(R * T), pi(R * T);
  for (int e = 0; e < R * T; ++e) { ri[e] = (int32_t)r_idx[e]; pi[e] = (int32_t)p_idx[e]; }

  // one allocation, 256-byte aligned sub-arrays
  struct Part { const void* src; size_t bytes; size_t off; };
  std::vector<Part> parts = {
      {ri.data(), ri.size() * 4, 0}, {pi.data(), pi.size() * 4, 0},
      {r_st, (size_t)R * T * 8, 0},  {p_st, (size_t)R * T * 8, 0},
      {three, (size_t)R, 0},         {sdesc.data(), sdesc.size() * 4, 0},
      {swi.data(), swi.size() * 4, 0}, {jp.data(), jp.size() * 4, 0},
      {jwi.data(), jwi.size() * 4, 0}, {coefs.data(), coefs.size() * 8, 0},
      {order.data(), order.size() * 4, 0}, {snp.data(), snp.size() * 4, 0}, {snw.data(), snw.size() * 4, 0}};
  size_t total = 0;
  for (auto& p : parts) { p.off = total; total += (p.bytes + 255) & ~(size_t)255; }
  void* base = nullptr;
  cudaError_t e = cudaMalloc(&base, total);
  if (e != cudaSuccess) return fail(VB_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  for (auto& p : parts) {
    e = cudaMemcpy((char*)base + p.off, p.src, p.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { cudaFree(base); return cuda_fail(e, "cudaMemcpy"); }
  }
  VbNet* net = new VbNet;
  net->tune = VbTuning{0, 0, 0, 1, 0, 0};
  char* b = (char*)base;
  vb::NetDev& d = net->dev;
  d.ni = ni; d.nr = nr; d.T = T;
  d.r_idx = (const int32_t*)(b + parts[0].off);
  d.p_idx = (const int32_t*)(b + parts[1].off);
  d.r_st = (const double*)(b + parts[2].off);
  d.p_st = (const double*)(b + parts[3].off);
  d.three = (const uint8_t*)(b + parts[4].off);
  d.sum_desc = (const uint2*)(b + parts[5].off);
  d.sum_w = (const uint32_t*)(b + parts[6].off);
  d.jac_ptr = (const int32_t*)(b + parts[7].off);
  d.jac_w = (const uint32_t*)(b + parts[8].off);
  d.coef_tab = (const double*)(b + parts[9].off);
  d.n_coef = (int)coefs.size();
  d.jac_desc = (const uint2*)(b + parts[10].off);
  d.sum_nptr = (const int32_t*)(b + parts[11].off);
  d.sum_nw = (const uint32_t*)(b + parts[12].off);
  net->base = base;
  net->bytes = total;
  *out = net;
  return VB_OK;
}

int vb_net_destroy(VbNet* net) {
  if (!net) return VB_OK;
  cudaError_t e = cudaFree(net->base);
  delete net;
  if (e != cudaSuccess) return cuda_fail(e, "cudaFree");
  return VB_OK;
}

size_t vb_net_device_bytes(const VbNet* net) { return net ? net->bytes : 0; }

int vb_net_set_tuning(VbNet* net, const VbTuning* t) {
  if (!net || !t) return fail(VB_ERR_ARG, "null argument");
  if (t->factor_kernel < 0 || t->factor_kernel > 4 || t->factor_ctas < 0 || t->factor_ctas > 2 ||
      t->sweep_stages < 0 || t->sweep_stages > 3 || t->streams < 0 || t->streams > 2 || t->stage1_layers < 0 ||
      t->stage1_layers > 2)
    return fail(VB_ERR_ARG, "tuning out of range (factor_kernel 0..4, factor_ctas 0..2, sweep_stages 0..3, "
                            "streams 0..2, stage1_layers 0..2)");
  net->tune = *t;
  return VB_OK;
}

int vb_net_get_tuning(const VbNet* net, VbTuning* t) {
  if (!net || !t) return fail(VB_ERR_ARG, "null argument");
  *t = net->tune;
  return VB_OK;
}

size_t vb_ros2_workspace_bytes(int batch, int nz, int ni, const int64_t* zoff_host) {
  int64_t layers = zoff_host ? zoff_host[batch] : (int64_t)batch * nz;
  return (size_t)layers * vb::ws_per_layer(ni, vb::round_even(ni)) * sizeof(double);
}

static vb::Batch make_batch(const VbNet* net, int batch, int nz, const int64_t* zoff) {
  vb::Batch B;
  B.count = batch;
  B.nz = nz;
  B.ni = net->dev.ni;
  B.nr = net->dev.nr;
  B.ld = vb::round_even(B.ni);
  B.zoff = zoff;
  B.factor_kernel = net->tune.factor_kernel;
  B.factor_ctas = net->tune.factor_ctas;
  B.sweep_stages = net->tune.sweep_stages;
  B.stage1_layers = net->tune.stage1_layers;
  return B;
}

// The launch sequence of one Ros2 step (jax_step.py:249-315) on one stream.
size_t vb_ros2_assembly_bytes(const VbNet* net, int batch, int nz) {
  if (!net || batch < 1 || nz < 1) return 0;
  return (size_t)batch * nz * vb::rates_region_doubles(net->dev.nr) * sizeof(double);
}

// The rate region of the layer-vectorized stage 2 in a vb_ros2_step
// workspace (after the step's own bytes, on a 256-byte boundary), or nullptr
// when the workspace does not hold it (the per-layer stage-2 kernel runs then).
static double* assembly_region(const VbNet* net, int batch, int nz, void* ws, size_t ws_bytes) {
  const size_t off = (vb_ros2_workspace_bytes(batch, nz, net->dev.ni, nullptr) + 255) & ~(size_t)255;
  const size_t need = vb_ros2_assembly_bytes(net, batch, nz);
  if (ws_bytes < off || ws_bytes - off < need) return nullptr;
  return reinterpret_cast<double*>(static_cast<char*>(ws) + off);
}

static int ros2_sequence(const VbNet* net, const vb::Batch& B, const double* y, const double* k, const double* dt,
                         const double* atm, int32_t flags, const uint8_t* fix_mask, double* sol, double* delta,
                         int32_t* status, double* ws, cudaStream_t st) {
  {
    ProfScope p(0, st);
    VB_CHECK(vb::launch_stage1(net->dev, B, y, k, dt, atm, flags, fix_mask, ws, st), "stage1");
  }
  {
    ProfScope p(1, st);
    VB_CHECK(vb::launch_factor(B, ws, status, 1, st), "factor");
  }
  vb::SweepArgs a{};
  a.mode = 1;
  a.status = status;
  {
    ProfScope p(2, st);
    VB_CHECK(vb::launch_sweep(B, ws, a, st), "back sweep 1");
  }
  {
    ProfScope p(3, st);
    VB_CHECK(vb::launch_stage2(net->dev, B, y, k, dt, atm, flags, fix_mask, ws, st), "stage2");
  }
  a.mode = 0;
  {
    ProfScope p(4, st);
    VB_CHECK(vb::launch_sweep(B, ws, a, st), "forward sweep 2");
  }
  a.mode = 2;
  a.y = y;
  a.sol = sol;
  a.delta = delta;
  {
    ProfScope p(5, st);
    VB_CHECK(vb::launch_sweep(B, ws, a, st), "back sweep 2");
  }
  return VB_OK;
}

// Second stream and fork / join events of the two-stream step, one set per
// device, created on first use.
namespace {
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
std::mutex g_side_mu;
SideStream g_side[kScratchDevices];
}  // namespace

static int side_stream(SideStream** out) {
  int dev = 0;
  VB_CHECK(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kScratchDevices) return fail(VB_ERR_ARG, "device ordinal beyond the stream table");
  std::lock_guard<std::mutex> lock(g_side_mu);
  SideStream& s = g_side[dev];
  if (!s.s) {
    VB_CHECK(cudaStreamCreateWithFlags(&s.s, cudaStreamNonBlocking), "cudaStreamCreate");
    VB_CHECK(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming), "cudaEventCreate");
    VB_CHECK(cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming), "cudaEventCreate");
  }
  *out = &s;
  return VB_OK;
}

int vb_ros2_step(const VbNet* net, int batch, int nz, const int64_t* zoff, const double* y, const double* k,
                 const double* dt, const double* atm, int32_t flags, const uint8_t* fix_mask, double* sol,
                 double* delta, int32_t* status, void* workspace, size_t ws_bytes, void* stream) {
  if (!net || !y || !k || !dt || !atm || !sol || !delta || !status || !workspace)
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2) return fail(VB_ERR_ARG, "batch >= 1 and nz >= 2 required");
  if (!zoff && ws_bytes < vb_ros2_workspace_bytes(batch, nz, net->dev.ni, nullptr))
    return fail(VB_ERR_ARG, "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  double* ws = (double*)workspace;
  double* rates = assembly_region(net, batch, nz, workspace, ws_bytes);
  VB_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * batch, st), "status reset");
  if (net->tune.streams != 2 || zoff || batch < 2) {
    vb::Batch B = make_batch(net, batch, nz, zoff);
    B.rates = rates;
    return ros2_sequence(net, B, y, k, dt, atm, flags, fix_mask, sol, delta, status, ws, st);
  }
  // two halves of a uniform batch, one per stream: the assembly of one half
  // overlaps the factor of the other (they bind different units of the SM)
  SideStream* side = nullptr;
  if (int rc = side_stream(&side)) return rc;
  const int h = batch / 2, ni = net->dev.ni, nr = net->dev.nr;
  const int64_t e = (int64_t)h * nz * ni;
  VB_CHECK(cudaEventRecord(side->fork, st), "fork");
  VB_CHECK(cudaStreamWaitEvent(side->s, side->fork, 0), "fork wait");
  vb::Batch B1 = make_batch(net, h, nz, nullptr), B2 = make_batch(net, batch - h, nz, nullptr);
  if (rates) {
    B1.rates = rates;
    B2.rates = rates + (int64_t)h * nz * vb::rates_region_doubles(nr);
  }
  if (int rc = ros2_sequence(net, B1, y, k, dt, atm, flags, fix_mask, sol, delta, status, ws, st)) return rc;
  if (int rc = ros2_sequence(net, B2, y + e, k + (int64_t)h * (nr + 1) * nz,
                             dt + h, atm + (int64_t)h * VB_ATM_DOUBLES(nz, ni), flags, fix_mask ? fix_mask + e : nullptr,
                             sol + e, delta + e, status + h,
                             ws + (int64_t)h * nz * vb::ws_per_layer(ni, vb::round_even(ni)), side->s))
    return rc;
  VB_CHECK(cudaEventRecord(side->join, side->s), "join");
  VB_CHECK(cudaStreamWaitEvent(st, side->join, 0), "join wait");
  return VB_OK;
}

// ---- mixed-precision step: workspace = FP64 step workspace, mixed region,
// per-atmosphere mode / todo / FP32 status / pass counters (256-byte aligned)
namespace {
struct MixedStepLayout {
  size_t mx, mode, todo, st32, npass, total;
};
MixedStepLayout mixed_step_layout(int batch, int nz, int ni) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const int64_t layers = (int64_t)batch * nz;
  MixedStepLayout m;
  m.mx = al(vb_ros2_workspace_bytes(batch, nz, ni, nullptr));
  m.mode = m.mx + al((size_t)layers * vb::mx_bytes_per_layer(ni));
  m.todo = m.mode + al((size_t)batch * 4);
  m.st32 = m.todo + al((size_t)batch * 4);
  m.npass = m.st32 + al((size_t)batch * 4);
  m.total = m.npass + al((size_t)batch * 4);
  return m;
}
}  // namespace

size_t vb_ros2_mixed_workspace_bytes(int batch, int nz, int ni, const int64_t* zoff_host) {
  if (batch < 1 || ni < 1) return 0;
  const int64_t layers = zoff_host ? zoff_host[batch] : (int64_t)batch * nz;
  const int nzs = (int)((layers + batch - 1) / batch);   // a ragged batch is sized by its layer total
  return mixed_step_layout(batch, zoff_host ? (nz > nzs ? nz : nzs) : nz, ni).total;
}

int vb_ros2_step_mixed(const VbNet* net, int batch, int nz, const int64_t* zoff, const double* y, const double* k,
                       const double* dt, const double* atm, int32_t flags, const uint8_t* fix_mask, int max_refine,
                       double tol, double* sol, double* delta, int32_t* status, int32_t* passes, void* workspace,
                       size_t ws_bytes, void* stream) {
  if (!net || !y || !k || !dt || !atm || !sol || !delta || !status || !workspace)
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2) return fail(VB_ERR_ARG, "batch >= 1 and nz >= 2 required");
  if (net->dev.ni > 96) return fail(VB_ERR_ARG, "the mixed-precision step supports ni <= 96");
  if (max_refine < 0 || max_refine > 8) return fail(VB_ERR_ARG, "max_refine must be in [0, 8]");
  if (!(tol > 0.0)) return fail(VB_ERR_ARG, "tol must be positive");
  const MixedStepLayout L = mixed_step_layout(batch, nz, net->dev.ni);
  if (ws_bytes < L.total)
    return fail(VB_ERR_ARG, "workspace too small (vb_ros2_mixed_workspace_bytes with zoff_host = NULL and nz = "
                            "the maximum layer count)");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = make_batch(net, batch, nz, zoff);
  char* base = (char*)workspace;
  // the optional rate region of the thread-per-layer stage 2, after the
  // mixed step's own bytes on a 256-byte boundary
  {
    const size_t off = (L.total + 255) & ~(size_t)255;
    if (ws_bytes >= off && ws_bytes - off >= vb_ros2_assembly_bytes(net, batch, nz))
      B.rates = reinterpret_cast<double*>(base + off);
  }
  double* ws = (double*)base;
  void* mxr = base + L.mx;
  int32_t* mode = (int32_t*)(base + L.mode);
  int32_t* todo = (int32_t*)(base + L.todo);
  int32_t* st32 = (int32_t*)(base + L.st32);
  int32_t* np = (int32_t*)(base + L.npass);
  VB_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * batch, st), "status reset");
  VB_CHECK(cudaMemsetAsync(st32, 0, sizeof(int32_t) * batch, st), "fp32 status reset");
  VB_CHECK(cudaMemsetAsync(np, 0, sizeof(int32_t) * batch, st), "passes reset");
  {
    ProfScope p(0, st);
    VB_CHECK(vb::launch_stage1(net->dev, B, y, k, dt, atm, flags, fix_mask, ws, st), "stage1");
  }
  {
    ProfScope p(1, st);
    VB_CHECK(vb::launch_factor32(B, ws, mxr, st32, st), "fp32 factor");
    VB_CHECK(vb::launch_mx_mode(batch, 0, mode, todo, st32, status, st), "modes");
    VB_CHECK(vb::launch_factor_only(B, ws, todo, status, st), "fp64 factor (fp32 failures)");
  }
  for (int stage = 0; stage < 2; ++stage) {
    if (stage == 1) {
      ProfScope p(3, st);
      VB_CHECK(vb::launch_stage2(net->dev, B, y, k, dt, atm, flags, fix_mask, ws, st), "stage2");
    }
    ProfScope p(stage == 0 ? 2 : 4, st);
    VB_CHECK(vb::launch_mx_pass(B, ws, mxr, stage, true, mode, nullptr, np, tol, status, st), "solve");
    for (int it = 0; it < max_refine; ++it)
      VB_CHECK(vb::launch_mx_pass(B, ws, mxr, stage, false, mode, nullptr, np, tol, status, st), "refinement");
    VB_CHECK(vb::launch_mx_mode(batch, 1, mode, todo, st32, status, st), "stall");
    VB_CHECK(vb::launch_factor_only(B, ws, todo, status, st), "fp64 factor (stalled)");
    VB_CHECK(vb::launch_mx_pass(B, ws, mxr, stage, true, mode, todo, np, tol, status, st), "fp64 solve");
  }
  {
    ProfScope p(5, st);
    VB_CHECK(vb::launch_mx_finish(B, ws, y, sol, delta, status, st), "sol and delta");
  }
  if (passes) VB_CHECK(cudaMemcpyAsync(passes, np, sizeof(int32_t) * batch, cudaMemcpyDeviceToDevice, st), "passes");
  return VB_OK;
}

int vb_ros2_stages(const VbNet* net, int batch, int nz, const int64_t* zoff, const void* workspace, double* k1,
                   double* k2, void* stream) {
  if (!net || !workspace) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2) return fail(VB_ERR_ARG, "batch >= 1 and nz >= 2 required");
  vb::Batch B = make_batch(net, batch, nz, zoff);
  VB_CHECK(vb::launch_gather_stages(B, (const double*)workspace, k1, k2, (cudaStream_t)stream), "stages");
  return VB_OK;
}

int vb_set_wait_limit(long long polls) {
  vb::set_wait_limit(polls);
  return VB_OK;
}

int vb_set_pipeline_wait_limit(long long polls) {
  vb::set_pipe_wait_limit(polls);
  return VB_OK;
}

int vb_set_factor_kernel(int variant) {
  if (variant < 0 || variant > 3) return fail(VB_ERR_ARG, "factor kernel variant must be 0, 1, 2 or 3");
  vb::set_factor_variant(variant);
  return VB_OK;
}

int vb_chem_rhs(const VbNet* net, int batch, int nz, const double* y, const double* M, const double* k,
                double* dydt, void* stream) {
  if (!net || !y || !M || !k || !dydt) return fail(VB_ERR_ARG, "null argument");
  VB_CHECK(vb::launch_chem(net->dev, batch, nz, y, M, k, dydt, nullptr, (cudaStream_t)stream), "chem_rhs");
  return VB_OK;
}

int vb_chem_jac(const VbNet* net, int batch, int nz, const double* y, const double* M, const double* k,
                double* jac, void* stream) {
  if (!net || !y || !M || !k || !jac) return fail(VB_ERR_ARG, "null argument");
  VB_CHECK(vb::launch_chem(net->dev, batch, nz, y, M, k, nullptr, jac, (cudaStream_t)stream), "chem_jac");
  return VB_OK;
}

int vb_diffusion(int batch, int nz, int ni, const double* y, const double* atm, int32_t flags, double* diff,
                 double* diag_d, double* sup_d, double* sub_d, void* stream) {
  if (!y || !atm) return fail(VB_ERR_ARG, "null argument");
  if (nz < 2 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "bad shape");
  VB_CHECK(vb::launch_diffusion(batch, nz, ni, y, atm, flags, diff, diag_d, sup_d, sub_d,
                                (cudaStream_t)stream),
           "diffusion");
  return VB_OK;
}

size_t vb_bt_factor_bytes(int batch, int nz, int ni) {
  return (size_t)batch * nz * vb::ws_per_layer(ni, vb::round_even(ni)) * sizeof(double);
}

static vb::Batch bt_batch(int batch, int nz, int ni) {
  vb::Batch B;
  B.count = batch; B.nz = nz; B.ni = ni; B.nr = 0; B.ld = vb::round_even(ni); B.zoff = nullptr;
  return B;
}

int vb_bt_factor(int batch, int nz, int ni, const double* diag, const double* sup_d, const double* sub_d,
                 void* factors, int32_t* status, void* stream) {
  if (!diag || !sup_d || !sub_d || !factors || !status) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 1 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "bad shape");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = bt_batch(batch, nz, ni);
  VB_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * batch, st), "status reset");
  VB_CHECK(vb::launch_pack_blocks(B, diag, sup_d, sub_d, (double*)factors, st), "pack");
  VB_CHECK(vb::launch_factor(B, (double*)factors, status, 0, st), "factor");
  return VB_OK;
}

static int bt_solve(int batch, int nz, int ni, const void* factors, const double* rhs, double* x, int trans,
                    void* stream) {
  if (!factors || !rhs || !x) return fail(VB_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = bt_batch(batch, nz, ni);
  if (x != rhs)
    VB_CHECK(cudaMemcpyAsync(x, rhs, sizeof(double) * batch * nz * ni, cudaMemcpyDeviceToDevice, st), "copy");
  vb::SweepArgs a{};
  a.transposed = trans;
  a.user = x;
  a.mode = 0;
  VB_CHECK(vb::launch_sweep(B, (double*)factors, a, st), "forward sweep");
  a.mode = 1;
  VB_CHECK(vb::launch_sweep(B, (double*)factors, a, st), "back sweep");
  return VB_OK;
}

int vb_bt_solve(int batch, int nz, int ni, const void* factors, const double* rhs, double* x, void* stream) {
  return bt_solve(batch, nz, ni, factors, rhs, x, 0, stream);
}

int vb_bt_solve_T(int batch, int nz, int ni, const void* factors, const double* rhs, double* x,
                  void* stream) {
  return bt_solve(batch, nz, ni, factors, rhs, x, 1, stream);
}

// ---- mixed-precision block solve: factors buffer layout (256-byte aligned parts)
namespace {
struct MixedLayout {
  size_t w64, inv32, inv64, state, fallback, passes, total;
};
MixedLayout mixed_layout(int batch, int nz, int ni) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t L = (size_t)batch * nz, blk = (size_t)ni * vb::round_even(ni);
  MixedLayout m;
  m.w64 = 0;
  m.inv32 = al(L * vb::ws_per_layer(ni, vb::round_even(ni)) * sizeof(double));
  // FP32 inverses: the row-equilibrated mixed region (X, row scales) for ni <= 96,
  // plain inverses of stride ld above
  const size_t f32 = std::max(L * blk * sizeof(float), (size_t)(L * vb::mx_bytes_per_layer(ni)));
  m.inv64 = m.inv32 + al(f32);
  m.state = m.inv64 + al(L * blk * sizeof(double));
  m.fallback = m.state + al((size_t)batch * 4);
  m.passes = m.fallback + al((size_t)batch * 4);
  m.total = m.passes + al((size_t)batch * 4);
  return m;
}
}  // namespace

size_t vb_bt_mixed_bytes(int batch, int nz, int ni) {
  if (batch < 1 || nz < 1 || ni < 1) return 0;
  return mixed_layout(batch, nz, ni).total;
}

int vb_bt_factor_mixed(int batch, int nz, int ni, const double* diag, const double* sup_d, const double* sub_d,
                       void* factors, int32_t* status, void* stream) {
  if (!diag || !sup_d || !sub_d || !factors || !status) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 1 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "bad shape");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = bt_batch(batch, nz, ni);
  const MixedLayout m = mixed_layout(batch, nz, ni);
  char* base = (char*)factors;
  VB_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * batch, st), "status reset");
  VB_CHECK(vb::launch_pack_blocks(B, diag, sup_d, sub_d, (double*)(base + m.w64), st), "pack");
  // up to 96 species: rows equilibrated by powers of two before the FP32
  // inversion (X = (R A')^{-1}, A'^{-1} = X diag(r)); above, plain FP32 inverses
  if (ni <= 96)
    VB_CHECK(vb::launch_factor32(B, (double*)(base + m.w64), base + m.inv32, status, st), "fp32 factor");
  else
    VB_CHECK(vb::launch_factor_into<float>(B, (double*)(base + m.w64), (float*)(base + m.inv32), nullptr, status,
                                           st),
             "fp32 factor");
  return VB_OK;
}

int vb_bt_solve_mixed(int batch, int nz, int ni, void* factors, const double* rhs, double* x, int max_refine,
                      double tol, int32_t* status, int32_t* passes, void* stream) {
  if (!factors || !rhs || !x || !status) return fail(VB_ERR_ARG, "null argument");
  if (x == rhs) return fail(VB_ERR_ARG, "x must not alias rhs");
  if (batch < 1 || nz < 1 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "bad shape");
  if (max_refine < 1 || max_refine > 8) return fail(VB_ERR_ARG, "max_refine must be in [1, 8]");
  if (!(tol > 0.0)) return fail(VB_ERR_ARG, "tol must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = bt_batch(batch, nz, ni);
  const MixedLayout m = mixed_layout(batch, nz, ni);
  char* base = (char*)factors;
  double* ws = (double*)(base + m.w64);
  int32_t* state = (int32_t*)(base + m.state);
  int32_t* fb = (int32_t*)(base + m.fallback);
  int32_t* np = (int32_t*)(base + m.passes);
  VB_CHECK(cudaMemsetAsync(state, 0, sizeof(int32_t) * batch, st), "state reset");
  VB_CHECK(cudaMemsetAsync(np, 0, sizeof(int32_t) * batch, st), "passes reset");
  const float* inv32 = (const float*)(base + m.inv32);
  const void* mxr = ni <= 96 ? (const void*)(base + m.inv32) : nullptr;   // equilibrated factors
  VB_CHECK(vb::launch_refine<float>(B, ws, inv32, mxr, rhs, x, state, np, tol, 1, nullptr, st), "fp32 solve");
  for (int it = 0; it < max_refine; ++it)
    VB_CHECK(vb::launch_refine<float>(B, ws, inv32, mxr, rhs, x, state, np, tol, 0, nullptr, st), "refinement");
  VB_CHECK(vb::launch_refine_finalize(batch, state, fb, status, st), "finalize");
  // FP64 fallback for the atmospheres whose refinement stalled (the others skip)
  double* inv64 = (double*)(base + m.inv64);
  VB_CHECK(vb::launch_factor_into<double>(B, ws, inv64, fb, status, st), "fp64 factor");
  VB_CHECK(vb::launch_refine<double>(B, ws, inv64, nullptr, rhs, x, state, np, tol, 1, fb, st), "fp64 solve");
  VB_CHECK(vb::launch_refine<double>(B, ws, inv64, nullptr, rhs, x, state, np, tol, 0, fb, st), "fp64 refinement");
  if (passes)
    VB_CHECK(cudaMemcpyAsync(passes, np, sizeof(int32_t) * batch, cudaMemcpyDeviceToDevice, st), "passes");
  return VB_OK;
}

int vb_residual(const VbNet* net, int batch, int nz, const int64_t* zoff, const double* y, const double* k,
                const double* atm, int32_t flags, double* f, void* stream) {
  if (!net || !y || !k || !atm || !f) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2) return fail(VB_ERR_ARG, "batch >= 1 and nz >= 2 required");
  vb::Batch B = make_batch(net, batch, nz, zoff);
  VB_CHECK(vb::launch_stage2(net->dev, B, y, k, nullptr, atm, flags, nullptr, nullptr, (cudaStream_t)stream, f),
           "residual");
  return VB_OK;
}

int vb_adjoint(const VbNet* net, int batch, int nz, const int64_t* zoff, const double* y, const double* k,
               const double* atm, int32_t flags, const double* v, double* lambda, double* g_k, double* g_M,
               double* g_Kzz, double* g_top, double* g_bot, double* g_vdep, int32_t* status, void* workspace,
               size_t ws_bytes, void* stream) {
  if (!net || !y || !k || !atm || !v || !status || !workspace) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2) return fail(VB_ERR_ARG, "batch >= 1 and nz >= 2 required");
  if (!zoff && ws_bytes < vb_ros2_workspace_bytes(batch, nz, net->dev.ni, nullptr))
    return fail(VB_ERR_ARG, "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = make_batch(net, batch, nz, zoff);
  double* ws = (double*)workspace;
  VB_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * batch, st), "status reset");
  VB_CHECK(vb::launch_stage1(net->dev, B, y, k, nullptr, atm, flags, nullptr, ws, st, v), "adjoint blocks");
  VB_CHECK(vb::launch_factor(B, ws, status, 0, st, true), "factor");
  vb::SweepArgs a{};
  a.transposed = 1;
  a.status = status;
  a.mode = 0;
  VB_CHECK(vb::launch_sweep(B, ws, a, st), "transposed forward sweep");
  a.mode = 1;
  VB_CHECK(vb::launch_sweep(B, ws, a, st), "transposed back sweep");
  // lambda is in the workspace's k1 rows
  VB_CHECK(vb::launch_gather_stages(B, ws, lambda, nullptr, st), "lambda");
  VB_CHECK(vb::launch_vjp(net->dev, B, y, k, atm, flags, ws, g_k, g_M, g_Kzz, g_top, g_bot, g_vdep, st), "vjp");
  return VB_OK;
}

int vb_photo_tau(int batch, int nz, int ni, const VbPhoto* photo, const double* y, const double* dz,
                 double* tau, void* stream) {
  if (!photo || !y || !dz || !tau) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || batch > 65535 || nz < 1 || ni < 1 || photo->nbin < 1) return fail(VB_ERR_ARG, "bad shape");
  VB_CHECK(vb::launch_photo_tau(batch, nz, ni, *photo, y, dz, tau, nullptr, nullptr, (cudaStream_t)stream), "photo tau");
  return VB_OK;
}

int vb_photo_flux(int batch, int nz, int ni, const VbPhoto* photo, const double* tau, const double* ymix,
                  const double* dflux_u_prev, double* aflux, double* sflux, double* dflux_d, double* dflux_u,
                  void* stream) {
  if (!photo || !tau || !ymix || !dflux_u_prev || !aflux || !sflux || !dflux_d || !dflux_u)
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || batch > 65535 || nz < 1 || ni < 1 || photo->nbin < 1) return fail(VB_ERR_ARG, "bad shape");
  VB_CHECK(vb::launch_photo_flux(batch, nz, ni, *photo, tau, ymix, dflux_u_prev, aflux, sflux, dflux_d, dflux_u,
                                 nullptr, 0.0, nullptr, (cudaStream_t)stream),
           "photo flux");
  return VB_OK;
}

int vb_photo_j(int batch, int nz, int nr, const VbPhoto* photo, const double* aflux, double* J_br,
               double* J_br_T, double* k, void* stream) {
  if (!photo || !aflux) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || batch > 65535 || nz < 1 || photo->nbin < 1 || photo->din12 < 0 || photo->din12 > photo->nbin)
    return fail(VB_ERR_ARG, "bad shape");
  VB_CHECK(vb::launch_photo_j(batch, nz, nr, *photo, aflux, J_br, J_br_T, k, nullptr, (cudaStream_t)stream),
           "photo J");
  return VB_OK;
}

int vb_photo_update(int batch, int nz, int ni, int nr, const VbPhoto* photo, const int32_t* due, const double* y,
                    const double* dz, const double* ymix, double* tau, double* aflux, double* sflux,
                    double* dflux_d, double* dflux_u, double* J_br, double* J_br_T, double* k, double flux_atol,
                    VbConvState* conv, void* stream) {
  if (!photo || !y || !dz || !ymix || !tau || !aflux || !sflux || !dflux_d || !dflux_u || !k)
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || batch > 65535 || nz < 1 || ni < 1 || nr < 1 || photo->nbin < 1 || photo->din12 < 0 || photo->din12 > photo->nbin)
    return fail(VB_ERR_ARG, "bad shape");
  cudaStream_t st = (cudaStream_t)stream;
  double* achg = conv ? &conv[0].aflux_change : nullptr;
  VB_CHECK(vb::launch_photo_tau(batch, nz, ni, *photo, y, dz, tau, due, achg, st), "photo tau");
  VB_CHECK(vb::launch_photo_flux(batch, nz, ni, *photo, tau, ymix, dflux_u, aflux, sflux, dflux_d, dflux_u, due,
                                 flux_atol, achg, st),
           "photo flux");
  VB_CHECK(vb::launch_photo_j(batch, nz, nr, *photo, aflux, J_br, J_br_T, k, due, st), "photo J");
  return VB_OK;
}

int vb_profile(int enable) {
  g_prof = enable != 0;
  return VB_OK;
}

int vb_profile_read(double* ms, int64_t* counts, int n) {
  if (n > VB_PROFILE_SITES) n = VB_PROFILE_SITES;
  for (int s = 0; s < VB_PROFILE_SITES; ++s) {
    double tot = 0.0;
    for (auto& pr : g_sites[s].ev) {
      cudaEventSynchronize(pr.second);
      float t = 0.f;
      cudaEventElapsedTime(&t, pr.first, pr.second);
      tot += t;
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    if (s < n) {
      if (ms) ms[s] = tot;
      if (counts) counts[s] = (int64_t)g_sites[s].ev.size();
    }
    g_sites[s].ev.clear();
  }
  return VB_OK;
}

int vb_rates(int batch, int nz, const VbRateTables* tables, const double* T, const double* M, int32_t flags,
             double* k, double* dkdT, void* stream) {
  if (!tables || !T || !M || !k) return fail(VB_ERR_ARG, "null argument");
  const VbRateTables& t = *tables;
  if (!t.code || !t.par || !t.nasa9 || !t.r_idx || !t.p_idx || !t.r_st || !t.p_st)
    return fail(VB_ERR_ARG, "null rate table");
  if (batch < 1 || batch > 65535 || nz < 1 || t.nr < 2 || (t.nr & 1) || t.nr / 2 > 65535 || t.ni < 1 ||
      t.max_terms < 1)
    return fail(VB_ERR_ARG, "bad shape: batch in [1, 65535], nz >= 1, nr even in [2, 131070], ni >= 1");
  VB_CHECK(vb::launch_rates(batch, nz, t, T, M, flags, k, dkdT, (cudaStream_t)stream), "rates");
  return VB_OK;
}

int vb_atm_refresh(int batch, int nz, int ni, const VbRefreshParams* params, const double* pico,
                   const double* mol_mass, const int32_t* esc_idx, const double* y, const double* ymix, double* atm,
                   double* mu, double* Hp, double* dz, double* zco, void* stream) {
  if (!params || !pico || !mol_mass || !y || !ymix || !atm || (params->n_esc > 0 && !esc_idx))
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2 || ni < 1 || params->n_esc < 0)
    return fail(VB_ERR_ARG, "batch >= 1, nz >= 2, ni >= 1, n_esc >= 0");
  if (params->pref_indx < 0 || params->pref_indx >= nz) return fail(VB_ERR_ARG, "pref_indx must be in [0, nz)");
  if ((5 * (size_t)nz + 1) * sizeof(double) > 200 * 1024) return fail(VB_ERR_ARG, "nz too large for the refresh");
  VB_CHECK(vb::launch_atm_refresh(batch, nz, ni, *params, pico, mol_mass, esc_idx, y, ymix, atm, mu, Hp, dz, zco,
                                  nullptr, 1, nullptr, (cudaStream_t)stream),
           "atm refresh");
  return VB_OK;
}

int vb_loop_refresh(int batch, int nz, int ni, const VbRefreshParams* params, int32_t update_frq,
                    const VbLoopScalars* scalars, const VbConvState* conv, const double* pico,
                    const double* mol_mass, const int32_t* esc_idx, const double* pre_y, const double* pre_ymix,
                    double* atm, double* mu, double* Hp, double* dz, double* zco, void* stream) {
  if (!params || !scalars || !pico || !mol_mass || !pre_y || !pre_ymix || !atm || (params->n_esc > 0 && !esc_idx))
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2 || ni < 1 || params->n_esc < 0)
    return fail(VB_ERR_ARG, "batch >= 1, nz >= 2, ni >= 1, n_esc >= 0");
  if (update_frq < 1) return fail(VB_ERR_ARG, "update_frq must be >= 1");
  if (params->pref_indx < 0 || params->pref_indx >= nz) return fail(VB_ERR_ARG, "pref_indx must be in [0, nz)");
  if ((5 * (size_t)nz + 1) * sizeof(double) > 200 * 1024) return fail(VB_ERR_ARG, "nz too large for the refresh");
  VB_CHECK(vb::launch_atm_refresh(batch, nz, ni, *params, pico, mol_mass, esc_idx, pre_y, pre_ymix, atm, mu, Hp, dz,
                                  zco, scalars, update_frq, conv, (cudaStream_t)stream),
           "loop refresh");
  return VB_OK;
}

int vb_conden_rates(int batch, int nz, int ni, int nr, int n_re, const int32_t* re_idx, const int32_t* sp_idx,
                    const double* coeff, const double* Dg, const double* sat_n, const double* y, double* k,
                    void* stream) {
  if (n_re == 0) return VB_OK;
  if (!re_idx || !sp_idx || !coeff || !Dg || !sat_n || !y || !k) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || batch > 65535 || nz < 1 || ni < 1 || nr < 2 || n_re < 0 || n_re > 65535)
    return fail(VB_ERR_ARG, "bad shape");
  VB_CHECK(vb::launch_conden_rates(batch, nz, ni, nr, n_re, re_idx, sp_idx, coeff, Dg, sat_n, y, k,
                                   (cudaStream_t)stream),
           "conden rates");
  return VB_OK;
}

int vb_conden_relax(int batch, int nz, int ni, const VbRelaxParams* params, const double* Dg, const double* sat,
                    const double* atm, const double* dt, double* y, double* ymix, void* stream) {
  if (!params || !Dg || !sat || !atm || !dt || !y || !ymix) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 1 || ni < 1) return fail(VB_ERR_ARG, "bad shape");
  const VbRelaxParams& p = *params;
  if (p.sp < 0 || p.sp >= ni || p.sp_l_s < 0 || p.sp_l_s >= ni || p.sp == p.sp_l_s)
    return fail(VB_ERR_ARG, "sp and sp_l_s must be distinct species in [0, ni)");
  VB_CHECK(vb::launch_conden_relax(batch, nz, ni, p, Dg, sat, atm, dt, y, ymix, (cudaStream_t)stream),
           "conden relax");
  return VB_OK;
}

int vb_loop_condense(int batch, int nz, int ni, int nr, const VbCondenLoop* conden, const VbLoopParams* params,
                     const double* atm, const uint8_t* gas_mask, const double* compo, const double* atom_ini,
                     const VbLoopScalars* scalars, const VbConvState* conv, const double* pre_td, double* pre_y,
                     double* pre_ymix, double* y, double* y_prev, double* ymix, double* atom_loss,
                     double* atom_loss_prev, double* k, void* stream) {
  if (!conden || !params || !atm || !compo || !atom_ini || !scalars || !pre_td || !pre_y || !pre_ymix || !y ||
      !y_prev || !ymix || !atom_loss || !atom_loss_prev || !k)
    return fail(VB_ERR_ARG, "null argument");
  const VbCondenLoop& c = *conden;
  if (batch < 1 || nz < 1 || ni < 1 || ni > VB_MAX_NI || nr < 2 || c.n_re < 0)
    return fail(VB_ERR_ARG, "bad shape");
  if (params->n_atoms < 1 || params->n_atoms > VB_LOOP_MAX_ATOMS) return fail(VB_ERR_ARG, "n_atoms must be in [1, 16]");
  if (c.n_re > 0 && (!c.re_idx || !c.sp_idx || !c.coeff || !c.Dg_re || !c.sat_re))
    return fail(VB_ERR_ARG, "condensation rows need re_idx, sp_idx, coeff, Dg_re and sat_re");
  if ((c.h2o_active && (!c.h2o_Dg || !c.h2o_sat)) || (c.nh3_active && (!c.nh3_Dg || !c.nh3_sat)))
    return fail(VB_ERR_ARG, "an active relaxation needs its Dg and saturation arrays");
  VB_CHECK(vb::launch_loop_condense(batch, nz, ni, nr, c, *params, atm, gas_mask, compo, atom_ini, scalars, conv,
                                    pre_td, pre_y, pre_ymix, y, y_prev, ymix, atom_loss, atom_loss_prev, k,
                                    (cudaStream_t)stream),
           "loop condensation");
  return VB_OK;
}

int vb_fp64_probe(double* out, int blocks, int threads, int iters, void* stream) {
  if (!out || blocks < 1 || threads < 32 || iters < 1) return fail(VB_ERR_ARG, "bad probe arguments");
  VB_CHECK(vb::launch_fp64_probe(out, blocks, threads, iters, (cudaStream_t)stream), "fp64 probe");
  return VB_OK;
}

int vb_loop_body(int batch, int nz, int ni, const int64_t* zoff, const VbLoopParams* params, const double* atm,
                 const uint8_t* gas_mask, const double* compo, const double* atom_ini, const uint8_t* fix_mask,
                 const double* fix_y, const double* sol, const double* delta_arr, double* y, double* y_prev,
                 double* ymix, double* atom_loss, double* atom_loss_prev, double* dt, VbLoopScalars* scalars,
                 const VbConvState* conv, double* pre_y, double* pre_ymix, double* pre_td, void* stream) {
  if ((pre_y == nullptr) != (pre_ymix == nullptr)) return fail(VB_ERR_ARG, "pre_y and pre_ymix go together");
  if (!params || !atm || !compo || !atom_ini || !sol || !delta_arr || !y || !y_prev || !ymix || !atom_loss ||
      !atom_loss_prev || !dt || !scalars)
    return fail(VB_ERR_ARG, "null argument");
  if ((fix_mask == nullptr) != (fix_y == nullptr)) return fail(VB_ERR_ARG, "fix_mask and fix_y go together");
  if (batch < 1 || nz < 2 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "batch >= 1, nz >= 2, 1 <= ni <= 128");
  const VbLoopParams& p = *params;
  if (p.n_atoms < 1 || p.n_atoms > VB_LOOP_MAX_ATOMS) return fail(VB_ERR_ARG, "n_atoms must be in [1, 16]");
  if ((p.flags & VB_LOOP_ADAPT_RTOL) && (p.adapt_rtol_dec_period < 1 || p.adapt_rtol_inc_period < 1))
    return fail(VB_ERR_ARG, "adaptive rtol periods must be >= 1");
  if (2 * (size_t)nz * sizeof(double) > 200 * 1024) return fail(VB_ERR_ARG, "nz too large for the loop body");
  vb::Batch B{};
  B.count = batch;
  B.nz = nz;
  B.ni = ni;
  B.ld = vb::round_even(ni);
  B.zoff = zoff;
  VB_CHECK(vb::launch_loop_body(B, p, gas_mask, compo, atom_ini, atm, fix_mask, fix_y, sol, delta_arr, y, y_prev,
                                ymix, atom_loss, atom_loss_prev, dt, scalars, conv, pre_y, pre_ymix, pre_td,
                                (cudaStream_t)stream),
           "loop body");
  return VB_OK;
}

int vb_loop_converge(int batch, int nz, int ni, const int64_t* zoff, const VbConvParams* params, const double* atm,
                     const double* slope_min, const uint8_t* ignore_mask, const double* y, const double* ymix,
                     const VbLoopScalars* scalars, double* ring_y, double* ring_t, VbConvState* conv,
                     int32_t* photo_due, void* stream) {
  if (!params || !atm || !slope_min || !y || !ymix || !scalars || !ring_y || !ring_t || !conv)
    return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "batch >= 1, nz >= 2, 1 <= ni <= 128");
  if (params->conv_step < 2) return fail(VB_ERR_ARG, "conv_step must be >= 2");
  vb::Batch B = bt_batch(batch, nz, ni);
  B.zoff = zoff;
  VB_CHECK(vb::launch_loop_conv(B, *params, atm, slope_min, ignore_mask, y, ymix, scalars, ring_y, ring_t, conv,
                                photo_due, (cudaStream_t)stream),
           "loop convergence");
  return VB_OK;
}

int vb_adjoint_atm(int batch, int nz, int ni, const int64_t* zoff, const double* y_star, const double* atm,
                   int32_t flags, const double* lambda, double* g_atm, void* stream) {
  if (!y_star || !atm || !lambda || !g_atm) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2 || ni < 1 || ni > VB_MAX_NI) return fail(VB_ERR_ARG, "batch >= 1, nz >= 2, 1 <= ni <= 128");
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = bt_batch(batch, nz, ni);
  B.zoff = zoff;
  const size_t total = zoff ? 0 : (size_t)batch * VB_ATM_DOUBLES(nz, ni);
  if (total) VB_CHECK(cudaMemsetAsync(g_atm, 0, total * sizeof(double), st), "clear");
  VB_CHECK(vb::launch_vjp_atm(B, y_star, atm, flags, lambda, g_atm, st), "vjp atm");
  return VB_OK;
}

int vb_ros2_step_static(const VbNet* net, int batch, int nz, const double* y, const double* k, const double* dt,
                        const double* atm, int32_t flags, const uint8_t* fix_mask, double* sol, double* delta,
                        int32_t* status, void* stream) {
  if (!net || !y || !k || !dt || !atm || !sol || !delta || !status) return fail(VB_ERR_ARG, "null argument");
  if (batch < 1 || nz < 2) return fail(VB_ERR_ARG, "batch >= 1 and nz >= 2 required");
  const size_t need = vb_ros2_workspace_bytes(batch, nz, net->dev.ni, nullptr);
  if (need > VB_STATIC_SCRATCH_BYTES)
    return fail(VB_ERR_ARG, "vb_ros2_step_static: batch needs " + std::to_string(need) +
                                " scratch bytes, above the static maximum of " +
                                std::to_string((size_t)VB_STATIC_SCRATCH_BYTES) +
                                " (use vb_ros2_step with a caller workspace)");
  double* ws = nullptr;
  if (int rc = static_scratch(&ws)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  vb::Batch B = make_batch(net, batch, nz, nullptr);
  // Every scratch value is written before it is read within the call, so
  // only the status words start at zero.
  VB_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * batch, st), "status reset");
  VB_CHECK(vb::launch_stage1(net->dev, B, y, k, dt, atm, flags, fix_mask, ws, st), "stage1");
  VB_CHECK(vb::launch_factor(B, ws, status, 1, st), "factor");
  vb::SweepArgs a{};
  a.mode = 1;
  a.status = status;
  VB_CHECK(vb::launch_sweep(B, ws, a, st), "back sweep 1");
  VB_CHECK(vb::launch_stage2(net->dev, B, y, k, dt, atm, flags, fix_mask, ws, st), "stage2");
  a.mode = 0;
  VB_CHECK(vb::launch_sweep(B, ws, a, st), "forward sweep 2");
  a.mode = 2;
  a.y = y;
  a.sol = sol;
  a.delta = delta;
  VB_CHECK(vb::launch_sweep(B, ws, a, st), "back sweep 2");
  return VB_OK;
}

}  // extern "C"
