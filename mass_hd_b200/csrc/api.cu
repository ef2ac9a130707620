// C ABI (include/mass_lb.h): handle lifetime, host <-> device transfers,
// step dispatch (FP64 unfused / FP32 fused / FP32 unfused for walls), the
// fused-kernel autotuner and the runtime-check reductions.
#include "mass_lb.h"
#include "mass_lb_ext.h"

#include "lb_common.cuh"
#include "unfused.h"
#include "fused32.cuh"
#include "reduce.cuh"
#include "stats.cuh"
#include "masks.cuh"

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

using namespace mlb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
  return fail(MASS_LB_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CU(call, where) do { const cudaError_t e_ = (call); \
  if(e_ != cudaSuccess) return cuda_fail(e_, where); } while(0)

const char* kFieldNames[MASS_LB_NUM_FIELDS] = {
  "ff", "QQxx", "QQyx", "phi", "n", "ux", "uy", "ux_phi", "uy_phi", "HHxx",
  "HHyx", "MU", "dxQQxx", "dyQQxx", "dxQQyx", "dyQQyx", "sigmaXX", "sigmaYY",
  "sigmaYX", "sigmaXY", "sigma_bulk", "sigma_elastic_xx", "sigma_elastic_yx",
  "sigma_phase_field_xx", "sigma_phase_field_yx", "sigma_active_xx",
  "sigma_active_yx", "fn", "QNxx", "QNyx", "phn", "m", "chi", "mN"};

constexpr long long kStageSites = 1ll << 24;   // sites per transfer chunk

// --------------------------------------------------------------------------
// host <-> device conversion kernels (one chunk of whole rows at a time)

// host AoS doubles [k][v] (k relative to chunk start) -> device planes
template<typename T>
__global__ void k_put_ff(const double* __restrict__ st, T* ff, long long plane,
                         int x0, int nrows, int LY, int g, int EY, double rest)
{
  const long long n = static_cast<long long>(nrows)*LY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    const int x = x0 + static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    const long long e = (y + g) + static_cast<long long>(EY)*(x + g);
#pragma unroll
    for(int v = 0; v < 9; ++v)
      ff[v*plane + e] = static_cast<T>(st[9*k + v] - Tv(v)*rest);
  }
}

template<typename T>
__global__ void k_get_ff(double* __restrict__ st, const T* ff, long long plane,
                         int x0, int nrows, int LY, int g, int EY, double rest)
{
  const long long n = static_cast<long long>(nrows)*LY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    const int x = x0 + static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    const long long e = (y + g) + static_cast<long long>(EY)*(x + g);
    // rest = 0 (FP64 planes hold the populations themselves): no add, so
    // that a -0 stays -0
#pragma unroll
    for(int v = 0; v < 9; ++v)
      st[9*k + v] = rest != 0.0 ? static_cast<double>(ff[v*plane + e]) + Tv(v)*rest
                                : static_cast<double>(ff[v*plane + e]);
  }
}

template<typename T>
__global__ void k_put_scalar(const double* __restrict__ st, T* a, int x0, int nrows,
                             int LY, int g, int EY)
{
  const long long n = static_cast<long long>(nrows)*LY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    const int x = x0 + static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    a[(y + g) + static_cast<long long>(EY)*(x + g)] = static_cast<T>(st[k]);
  }
}

template<typename T>
__global__ void k_get_scalar(double* __restrict__ st, const T* a, int x0, int nrows,
                             int LY, int g, int EY, double add)
{
  const long long n = static_cast<long long>(nrows)*LY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    const int x = x0 + static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    const double v = static_cast<double>(a[(y + g) + static_cast<long long>(EY)*(x + g)]);
    st[k] = add != 0.0 ? v + add : v;   // keeps the sign of a zero
  }
}

// chi = m/phi (0 where phi <= 1e-12) from the fused go-or-grow planes, in
// FP32 as the unfused sweeps store it (src/models/go-or-grow.cpp:208-216)
__global__ void k_get_chi(double* __restrict__ st, const float* phi, const float* m, int x0,
                          int nrows, int LY)
{
  const long long n = static_cast<long long>(nrows)*LY;
  const long long base = static_cast<long long>(x0)*LY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    const float p = phi[base + k];
    st[k] = p > 1e-12f ? static_cast<double>(m[base + k]/p) : 0.0;
  }
}

inline int blocks_for(long long n)
{
  long long b = (n + 255)/256;
  return static_cast<int>(std::min<long long>(std::max<long long>(b, 1), 4096));
}

// ---- wall bands of a fused lattice ----------------------------------------
// A fused FP32 lattice with walls steps in two parts. The warp-strip kernel
// (and, with npc > 1, the corrector sub-steps after it) steps the whole
// lattice as if it were periodic. One Step() reaches
// keep = 2 + 2*npc sites (predictor UpdateQuantities, UpdateFields and
// Move, then UpdateQuantities and UpdateFields per corrector), so every site
// at least `keep` sites from a wall gets exactly what the wall step gives
// it: its dependence cone holds no ghost value and no site whose update a
// wall changes. The sites nearer a wall come from a band lattice: the
// half = 2*keep rows next to each wall of one axis, side by side, stepped
// by the wall-aware sweeps (step_unfused_f32) with the lattice's own
// boundary kind. The band's outer `keep` rows on each side are exact; the
// cut between its halves reaches only rows that are discarded. Channels
// (walls across y) take one band of LX x 2*half sites, boxes a second of
// 2*half x LY.
struct BandMap
{
  int axis;            // 0: the band crosses y (walls front/back), 1: crosses x
  int LX, LY;          // the whole lattice
  int BX, BY;          // the band's sites
  int EY;              // the band's extended row (BY + 2, ghost ring g = 1)
  long long NE;        // the band's extended plane
  long long plane;     // LX*LY, the fused plane
  int half, keep;      // rows taken next to each wall, rows kept
};

// band planes: ff (9 planes), the scalars Qxx, Qyx, [phi], [m] in the fused
// plane order 9, 10, 11, 12, and the phi source rate
struct BandPtrs
{
  float* ff;
  float* sc[4];
  int nsc;
  float* src;
  const float* src_fused;
};

// the band's derived planes in the fused diagnostic order (fields n ..
// sigma_active_yx); null where the model has none
struct BandDiag
{
  const float* a[NDIAG];
  float rho;
};

__device__ __forceinline__ int band_row(const BandMap& m, int i, int N)
{
  return i < m.half ? i : N - 2*m.half + i;
}

// band site k -> fused index gi, band extended index bi; keep: the site is
// one of the rows the band step leaves exact
__device__ __forceinline__ bool band_site(const BandMap& m, long long k, long long& gi,
                                          long long& bi)
{
  const int bx = static_cast<int>(k / m.BY), by = static_cast<int>(k % m.BY);
  const int x = m.axis == 1 ? band_row(m, bx, m.LX) : bx;
  const int y = m.axis == 0 ? band_row(m, by, m.LY) : by;
  gi = static_cast<long long>(x)*m.LY + y;
  bi = static_cast<long long>(bx + 1)*m.EY + (by + 1);
  const int r = m.axis == 0 ? by : bx;
  return r < m.keep || r >= 2*m.half - m.keep;
}

__global__ void __launch_bounds__(256)
k_band_gather(BandMap m, const float* __restrict__ from, BandPtrs p)
{
  const long long n = static_cast<long long>(m.BX)*m.BY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    long long gi, bi;
    band_site(m, k, gi, bi);
#pragma unroll
    for(int v = 0; v < 9; ++v) p.ff[v*m.NE + bi] = from[v*m.plane + gi];
    for(int i = 0; i < p.nsc; ++i) p.sc[i][bi] = from[(9 + i)*m.plane + gi];
    if(p.src) p.src[bi] = p.src_fused[gi];
  }
}

__global__ void __launch_bounds__(256)
k_band_scatter(BandMap m, float* __restrict__ to, BandPtrs p)
{
  const long long n = static_cast<long long>(m.BX)*m.BY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    long long gi, bi;
    if(!band_site(m, k, gi, bi)) continue;
#pragma unroll
    for(int v = 0; v < 9; ++v) to[v*m.plane + gi] = p.ff[v*m.NE + bi];
    for(int i = 0; i < p.nsc; ++i) to[(9 + i)*m.plane + gi] = p.sc[i][bi];
  }
}

__global__ void __launch_bounds__(256)
k_band_diag(BandMap m, float* __restrict__ diag, BandDiag d)
{
  const long long n = static_cast<long long>(m.BX)*m.BY;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < n; k += 256ll*gridDim.x)
  {
    long long gi, bi;
    if(!band_site(m, k, gi, bi)) continue;
    // the fused diagnostics hold the density n, the sweeps its deviation
    if(d.a[0]) diag[gi] = d.rho + d.a[0][bi];
    for(int p = 1; p < NDIAG; ++p)
      if(d.a[p]) diag[p*m.plane + gi] = d.a[p][bi];
  }
}

struct WallBand
{
  BandMap map{};
  Dims d{};
  State<float> s{};
  float* src = nullptr;   // the phi source rate on the band's extended torus
};

} // namespace

// --------------------------------------------------------------------------

struct mass_lb_handle
{
  int device = 0;
  int precision = MASS_LB_FP64;
  int model = LYO;
  unsigned LX = 0, LY = 0, bc = 0;
  int wall = 0;              // 1 if the lattice carries a ghost ring
  Params P{};
  Dims d{};
  cudaStream_t stream = nullptr;
  // Host<->device transfers of whole fields run on `xfer`, a stream of the
  // device's highest priority, forked from `stream` and joined back to it by
  // two events, so that their conversion kernels take the SMs ahead of other
  // handles' queued steps. `io` is the stream the transfer code issues on:
  // `xfer` inside an XferScope, `stream` elsewhere.
  cudaStream_t xfer = nullptr;
  cudaEvent_t xfer_in = nullptr, xfer_out = nullptr;
  cudaStream_t io = nullptr;
  cudaEvent_t order_ev = nullptr;   // mass_lb_stream_wait's mark on this stream
  bool fused = false;
  bool in_ensemble = false;  // a run of a mass_lb_ensemble (its buffers step there)

  State<double> s64{};       // FP64 (any bc)
  State<float> s32{};        // FP32 with walls
  std::vector<void*> allocs;

  // FP32 fused periodic state: NP planes each, ping-pong
  float* cur = nullptr;
  float* nxt = nullptr;
  float* diag = nullptr;     // NDIAG planes, allocated on first use
  float* pred = nullptr;     // FP32 fused with npc > 1: fn, QNxx, QNyx[, phn] of the step
  float* scratch = nullptr;  // its derived-field replay's throw-away outputs (NP planes)
  bool diag_n_dev = false;   // the diagnostic n plane holds the density deviation
  unsigned step_x0 = 0, step_nx = 0;   // fused: the rows a step writes (0 rows: all)
  WallBand band[2];          // FP32 fused with walls: the band lattices
  int nbands = 0;
  cudaStream_t bstream[2] = {};     // their work beside the fused kernel
  cudaEvent_t band_in = nullptr, band_read[2] = {}, band_out[2] = {};
  bool has_prev = false;     // nxt holds the state before the last step
  bool derived_pending = false;   // unfused: the derived planes await replay_derived
  FusedConfig cfg{128, 256};
  bool tuned = false;

  double* stage = nullptr;   // device staging (kStageSites*9 doubles)
  StatScratch stats{};       // statistics scratch, allocated on first use
  double* red_scratch = nullptr;
  double* red_out = nullptr; // 3 doubles
  int* err = nullptr;

  double ftot = 0, ptot = 0;
  double* tot_host = nullptr;   // pinned: the sums of an asynchronous upload
  cudaEvent_t tot_ev = nullptr; // they have landed
  bool tot_pending = false;     // ftot/ptot still to be read from tot_host
  unsigned long long steps = 0;

  // division-model hooks (mass_lb_set_phi_source / _conservation)
  float* src_fused = nullptr;   // FP32 fused: rate plane of LX*LY
  double* src64 = nullptr;      // FP64: rate on the extended torus
  float* src32 = nullptr;       // FP32 with walls: same
  bool src_on = false;
  double* phisum = nullptr;     // countphi scalar for conserve_phi
  double* relaxsum = nullptr;   // relaxed phi total (go-or-grow)

  // device-side division / death masks (mass_lb_mask_candidates, _draw_mask)
  MaskScratch mk{};
  long long mk_count = -1;      // candidates of the last count, -1: none
  double* mk_pinned = nullptr;  // pinned host staging of the draws
  long long mk_pinned_cap = 0;
  cudaEvent_t mk_copied = nullptr;   // the last staging copy has been read

  // queued uniforms (mass_lb_mask_supply / mass_lb_draw_masks_queued)
  static constexpr int MQ_STAGES = 2;    // pinned staging buffers, used in turn
  static constexpr int MQ_SLOTS = 4;     // queued draws whose counts may be in flight
  MaskQueue mq{};
  double* mq_pinned[MQ_STAGES] = {};     // staging of supplied draws
  long long mq_pinned_cap[MQ_STAGES] = {};
  cudaEvent_t mq_copied[MQ_STAGES] = {}; // the last copy from each buffer has been read
  int mq_stage = 0;                      // the buffer of the next supply
  cudaStream_t mq_copy = nullptr;        // the supplies' copies (off the step stream)
  long long* mq_state = nullptr;         // device: [0] queue head, [1] error flag (low word)
  int* mq_err = nullptr;                 // the error flag as the kernels set it
  long long* mq_snap = nullptr;          // device: (head, flag) after each draw slot's draw
  long long* mq_host = nullptr;          // pinned: the same, per slot
  cudaEvent_t mq_drew[MQ_SLOTS] = {};    // a slot's draw has finished (step stream)
  cudaEvent_t mq_counted[MQ_SLOTS] = {}; // a slot's snapshot has landed
  long long mq_issued = 0;               // queued draws issued
  long long mq_known = 0;                // draws whose counts have been read (a prefix)
  long long mq_consumed = 0;             // draws consumed up to the last known draw
};

namespace {

struct DeviceGuard
{
  int prev = -1;
  explicit DeviceGuard(int dev)
  {
    cudaGetDevice(&prev);
    if(prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard()
  {
    int now = -1;
    cudaGetDevice(&now);
    if(prev >= 0 && now != prev) cudaSetDevice(prev);
  }
};

template<typename T>
int dalloc(mass_lb_handle* h, T** p, size_t n)
{
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, n*sizeof(T) > 0 ? n*sizeof(T) : 1);
  if(e != cudaSuccess)
  {
    cudaGetLastError();
    return fail(MASS_LB_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return 0;
}

// planes of the FP32 fused state: g0..g8, Qxx, Qyx, then phi (lyotropic,
// go-or-grow) and m (go-or-grow)
int nplanes(const mass_lb_handle* h) { return h->model == NEM ? 11 : h->model == LYO ? 12 : 13; }

template<typename T>
int alloc_state(mass_lb_handle* h, State<T>& s, const Dims& d)
{
  const size_t NE = static_cast<size_t>(d.NE);
  T** lb[4] = {&s.ff, &s.fn, &s.ff_tmp, &s.fn_tmp};
  for(auto p : lb) if(int r = dalloc(h, p, 9*NE)) return r;
  std::vector<T**> sc = {&s.Qxx, &s.Qyx, &s.Qxx_tmp, &s.Qyx_tmp, &s.QNxx, &s.QNyx, &s.n, &s.ux, &s.uy,
                         &s.Hxx, &s.Hyx, &s.dxQxx, &s.dyQxx, &s.dxQyx, &s.dyQyx,
                         &s.sXX, &s.sYY, &s.sYX, &s.sXY};
  if(h->model != NEM)
  {
    T** extra[6] = {&s.phi, &s.phn, &s.phi_tmp, &s.uxp, &s.uyp, &s.MU};
    for(int i = 0; i < 6; ++i) sc.push_back(extra[i]);
    for(int i = 0; i < 7; ++i) sc.push_back(&s.diag[i]);
  }
  if(h->model == GOG)
  {
    T** extra[5] = {&s.m, &s.mN, &s.m_tmp, &s.chi, &s.chi_tmp};
    for(int i = 0; i < 5; ++i) sc.push_back(extra[i]);
  }
  for(auto p : sc) if(int r = dalloc(h, p, NE)) return r;
  return 0;
}

template<typename T>
int zero_state(mass_lb_handle* h, State<T>& s, const Dims& d)
{
  const size_t NE = static_cast<size_t>(d.NE);
  T* lb[4] = {s.ff, s.fn, s.ff_tmp, s.fn_tmp};
  for(T* p : lb) CU(cudaMemsetAsync(p, 0, 9*NE*sizeof(T), h->stream), "memset");
  std::vector<T*> sc = {s.Qxx, s.Qyx, s.Qxx_tmp, s.Qyx_tmp, s.QNxx, s.QNyx, s.n, s.ux, s.uy, s.Hxx, s.Hyx,
                        s.dxQxx, s.dyQxx, s.dxQyx, s.dyQyx, s.sXX, s.sYY, s.sYX, s.sXY};
  if(h->model != NEM)
  {
    T* extra[6] = {s.phi, s.phn, s.phi_tmp, s.uxp, s.uyp, s.MU};
    for(int i = 0; i < 6; ++i) sc.push_back(extra[i]);
    for(int i = 0; i < 7; ++i) sc.push_back(s.diag[i]);
  }
  if(h->model == GOG)
  {
    T* extra[5] = {s.m, s.mN, s.m_tmp, s.chi, s.chi_tmp};
    for(int i = 0; i < 5; ++i) sc.push_back(extra[i]);
  }
  for(T* p : sc) CU(cudaMemsetAsync(p, 0, NE*sizeof(T), h->stream), "memset");
  return 0;
}

template<typename T>
int alloc_state(mass_lb_handle* h, State<T>& s) { return alloc_state(h, s, h->d); }
template<typename T>
int zero_state(mass_lb_handle* h, State<T>& s) { return zero_state(h, s, h->d); }

// FP32 parameters of the fused kernels (the same rounding for single
// lattices and ensemble runs, so both step bit-identically)
P32 p32_of(const Params& P)
{
  return P32{static_cast<float>(P.rho), static_cast<float>(P.GammaQ),
             static_cast<float>(P.GammaP), static_cast<float>(P.xi),
             static_cast<float>(P.tauNem), static_cast<float>(P.tauIso),
             static_cast<float>(P.friction), static_cast<float>(P.AA),
             static_cast<float>(P.CC), static_cast<float>(P.LL),
             static_cast<float>(P.KK), static_cast<float>(P.zeta),
             static_cast<float>(P.zetaI), static_cast<float>(P.conc),
             0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0};
}

// the same with the go-or-grow phenotype terms
P32 p32_of(const Params& P, const Pheno& ph)
{
  P32 q = p32_of(P);
  q.B = static_cast<float>(ph.B); q.Snem = static_cast<float>(ph.Snem);
  q.Dchi = static_cast<float>(ph.Dchi); q.Achi = static_cast<float>(ph.Achi);
  q.Ochi = static_cast<float>(ph.Ochi); q.phiswitch = static_cast<float>(ph.phiswitch);
  q.phi_critical = static_cast<float>(ph.phi_critical); q.growTogether = ph.growTogether;
  return q;
}

FusedArgs fused_args(mass_lb_handle* h, const float* in, float* out, bool diag)
{
  FusedArgs a{};
  a.in = in;
  a.out = out;
  a.diag = diag ? h->diag : nullptr;
  a.err = h->err;
  a.LX = static_cast<int>(h->LX);
  a.LY = static_cast<int>(h->LY);
  a.plane = static_cast<long long>(h->LX)*h->LY;
  a.p = h->model == GOG ? p32_of(h->P, h->s32.ph) : p32_of(h->P);
  // go-or-grow always reads its growth-rate plane (zero until a source is set)
  a.src = h->src_on || h->model == GOG ? h->src_fused : nullptr;
  a.pred = !diag && h->P.npc > 1 ? h->pred : nullptr;
  a.xbase = static_cast<int>(h->step_x0);
  a.xcount = static_cast<int>(h->step_nx ? h->step_nx : h->LX);
  return a;
}

// Lattices the CTA-strip kernel cannot step: a phi source, go-or-grow and
// npc > 1 are in the warp-strip kernel only.
bool warp_strip_only(const mass_lb_handle* h)
{
  return h->src_on || h->model == GOG || h->P.npc > 1;
}

// A further corrector (npc > 1) of a fused periodic lattice, `in` -> `out`:
// the sweeps' corrector sub-step on a view of the fused planes (they agree
// plane for plane with the sweeps' periodic layout) and of the predictor
// values the warp-strip kernel wrote. With `diag` it also writes the
// derived fields of its UpdateQuantities into the diagnostic planes.
int extra_corrector(mass_lb_handle* h, const float* in, float* out, bool diag)
{
  const long long p = static_cast<long long>(h->LX)*h->LY;
  State<float> v{};
  v.ff = const_cast<float*>(in);
  v.Qxx = const_cast<float*>(in) + 9*p;
  v.Qyx = const_cast<float*>(in) + 10*p;
  v.fn = h->pred;
  v.QNxx = h->pred + 9*p;
  v.QNyx = h->pred + 10*p;
  v.ff_tmp = out;
  v.Qxx_tmp = out + 9*p;
  v.Qyx_tmp = out + 10*p;
  if(h->model != NEM)
  {
    v.phi = const_cast<float*>(in) + 11*p;
    v.phn = h->pred + 11*p;
    v.phi_tmp = out + 11*p;
    v.src = h->src_on ? h->src_fused : nullptr;
  }
  if(diag)
  {
    // the fused diagnostic plane order (fields n .. sigma_active_yx)
    float* g = h->diag;
    v.n = g; v.ux = g + p; v.uy = g + 2*p; v.Hxx = g + 5*p; v.Hyx = g + 6*p;
    v.dxQxx = g + 8*p; v.dyQxx = g + 9*p; v.dxQyx = g + 10*p; v.dyQyx = g + 11*p;
    v.sXX = g + 12*p; v.sYY = g + 13*p; v.sYX = g + 14*p; v.sXY = g + 15*p;
    if(h->model != NEM)
    {
      v.uxp = g + 3*p; v.uyp = g + 4*p; v.MU = g + 7*p;
      for(int k = 0; k < 7; ++k) v.diag[k] = g + (16 + k)*p;
    }
  }
  // the fused planes carry no ghost ring, walls or not: a periodic view
  const int LX = static_cast<int>(h->LX), LY = static_cast<int>(h->LY);
  const Dims d{LX, LY, 0, LX, LY, p};
  if(corrector_substep_f32(d, h->P, v, diag, h->stream) != 0)
    return cuda_fail(cudaGetLastError(), "corrector");
  return 0;
}

// Moves an FP32 fused state into the unfused sweeps' state (allocated on
// first use) or back. The layouts agree plane for plane on a periodic
// lattice (no ghost ring, populations as deviations in both), so each is a
// device copy. The sweeps take over where the fused kernel cannot run: the
// dry relaxation of go-or-grow's Configure() and conserve_phi.
// One LX x LY plane between the fused layout (x*LY + y) and the sweeps'
// extended torus ((x+g)*EY + y + g); with walls (g = 1) the ghost ring is
// left to the boundary kernels of the next step.
cudaError_t plane_copy(const mass_lb_handle* h, float* dst, const float* src, bool to_sweeps)
{
  const Dims& d = h->d;
  const size_t row = static_cast<size_t>(d.LY)*sizeof(float);
  if(d.g == 0)
    return cudaMemcpyAsync(dst, src, row*d.LX, cudaMemcpyDeviceToDevice, h->stream);
  const long long off = static_cast<long long>(d.g)*d.EY + d.g;
  const size_t ext = static_cast<size_t>(d.EY)*sizeof(float);
  return to_sweeps
    ? cudaMemcpy2DAsync(dst + off, ext, src, row, row, d.LX, cudaMemcpyDeviceToDevice, h->stream)
    : cudaMemcpy2DAsync(dst, row, src + off, ext, row, d.LX, cudaMemcpyDeviceToDevice, h->stream);
}

int fused_to_sweeps(mass_lb_handle* h)
{
  if(!h->fused) return 0;
  if(!h->s32.ff)
  {
    if(int r = alloc_state(h, h->s32)) return r;
    if(int r = zero_state(h, h->s32)) return r;
  }
  const long long plane = static_cast<long long>(h->LX)*h->LY;
  State<float>& s = h->s32;
  for(int v = 0; v < 9; ++v)
    CU(plane_copy(h, s.ff + v*h->d.NE, h->cur + v*plane, true), "state copy");
  CU(plane_copy(h, s.Qxx, h->cur + 9*plane, true), "state copy");
  CU(plane_copy(h, s.Qyx, h->cur + 10*plane, true), "state copy");
  if(h->model != NEM) CU(plane_copy(h, s.phi, h->cur + 11*plane, true), "state copy");
  if(h->model == GOG) CU(plane_copy(h, s.m, h->cur + 12*plane, true), "state copy");
  if(h->src_on && h->src_fused)
  {
    if(!h->src32)
    {
      if(int r = dalloc(h, &h->src32, h->d.NE)) return r;
      CU(cudaMemsetAsync(h->src32, 0, h->d.NE*sizeof(float), h->stream), "memset");
    }
    CU(plane_copy(h, h->src32, h->src_fused, true), "copy");
    s.src = h->src32;
  }
  if(h->model == GOG && update_chi_f32(h->d, s, h->stream))
    return cuda_fail(cudaGetLastError(), "chi update");
  h->fused = false;
  h->has_prev = false;
  h->derived_pending = false;
  return 0;
}

int sweeps_to_fused(mass_lb_handle* h)
{
  if(h->fused) return 0;
  const long long plane = static_cast<long long>(h->LX)*h->LY;
  const State<float>& s = h->s32;
  for(int v = 0; v < 9; ++v)
    CU(plane_copy(h, h->cur + v*plane, s.ff + v*h->d.NE, false), "state copy");
  CU(plane_copy(h, h->cur + 9*plane, s.Qxx, false), "state copy");
  CU(plane_copy(h, h->cur + 10*plane, s.Qyx, false), "state copy");
  if(h->model != NEM) CU(plane_copy(h, h->cur + 11*plane, s.phi, false), "state copy");
  if(h->model == GOG) CU(plane_copy(h, h->cur + 12*plane, s.m, false), "state copy");
  h->fused = true;
  h->has_prev = false;
  h->derived_pending = false;
  return 0;
}

// ---- wall bands (the scheme is described above k_band_gather) -------------

bool walls_box(const mass_lb_handle* h)
{
  return h->model != NEM && (h->bc == 3 || h->bc == 4);
}

// rows one step reaches (the band rows kept) and rows taken per wall
int band_keep(const mass_lb_handle* h) { return 2 + 2*static_cast<int>(h->P.npc); }
int band_half(const mass_lb_handle* h) { return 2*band_keep(h); }

// the bands need two disjoint halves on every walled axis
bool bands_fit(const mass_lb_handle* h)
{
  const unsigned n = 2u*band_half(h);
  return h->LY >= n && (!walls_box(h) || h->LX >= n);
}

int init_bands(mass_lb_handle* h)
{
  h->nbands = walls_box(h) ? 2 : 1;
  int least = 0, greatest = 0;
  CU(cudaDeviceGetStreamPriorityRange(&least, &greatest), "priorities");
  CU(cudaEventCreateWithFlags(&h->band_in, cudaEventDisableTiming), "event");
  for(int i = 0; i < h->nbands; ++i)
  {
    CU(cudaStreamCreateWithPriority(&h->bstream[i], cudaStreamNonBlocking, greatest),
       "band stream");
    CU(cudaEventCreateWithFlags(&h->band_read[i], cudaEventDisableTiming), "event");
    CU(cudaEventCreateWithFlags(&h->band_out[i], cudaEventDisableTiming), "event");
  }
  const int LX = static_cast<int>(h->LX), LY = static_cast<int>(h->LY);
  const int half = band_half(h), keep = band_keep(h);
  for(int i = 0; i < h->nbands; ++i)
  {
    WallBand& b = h->band[i];
    const int BX = i == 0 ? LX : 2*half, BY = i == 0 ? 2*half : LY;
    b.d = Dims{BX, BY, 1, BX + 2, BY + 2, static_cast<long long>(BX + 2)*(BY + 2)};
    b.map = BandMap{i, LX, LY, BX, BY, BY + 2, b.d.NE, static_cast<long long>(LX)*LY, half, keep};
    if(int r = alloc_state(h, b.s, b.d)) return r;
    if(int r = zero_state(h, b.s, b.d)) return r;
    if(h->model != NEM)
    {
      if(int r = dalloc(h, &b.src, b.d.NE)) return r;
      CU(cudaMemsetAsync(b.src, 0, b.d.NE*sizeof(float), h->stream), "memset");
    }
  }
  return 0;
}

BandPtrs band_ptrs(const mass_lb_handle* h, const WallBand& b)
{
  BandPtrs p{};
  p.ff = b.s.ff;
  p.sc[0] = b.s.Qxx;
  p.sc[1] = b.s.Qyx;
  p.nsc = 2;
  if(h->model != NEM) p.sc[p.nsc++] = b.s.phi;
  if(h->model == GOG) p.sc[p.nsc++] = b.s.m;
  // the fused go-or-grow step reads a zero rate plane when no source is
  // set, the sweeps none: both leave phi as it is
  p.src = h->src_on && h->src_fused ? b.src : nullptr;
  p.src_fused = h->src_fused;
  return p;
}

// Band i's part of one step of a fused lattice with walls, on stream `st`:
// gather it from the state `from` (event band_read[i] marks the end of the
// reads), then step it with the walls. The step also keeps the derived
// fields of its last UpdateQuantities, which a download of derived fields
// scatters (band_emit with diag) without stepping again.
int band_compute(mass_lb_handle* h, int i, const float* from, cudaStream_t st)
{
  WallBand& b = h->band[i];
  const int nb = blocks_for(static_cast<long long>(b.map.BX)*b.map.BY);
  const BandPtrs p = band_ptrs(h, b);
  k_band_gather<<<nb, 256, 0, st>>>(b.map, from, p);
  CU(cudaGetLastError(), "band gather");
  CU(cudaEventRecord(h->band_read[i], st), "band gather");
  b.s.src = p.src;
  b.s.conserve_phi = 0;
  b.s.phisum = nullptr;
  b.s.ph = h->s32.ph;
  if(h->model == GOG && update_chi_f32(b.d, b.s, st))
    return cuda_fail(cudaGetLastError(), "band chi");
  if(step_unfused_f32(b.d, h->P, b.s, static_cast<int>(h->bc), 1, true, st) != 0)
    return cuda_fail(cudaGetLastError(), "band step");
  return 0;
}

// Then, on stream `st`: the bands' exact rows into the state `to` or, with
// `diag`, their derived fields into the diagnostic planes (whose n plane
// holds the density, or its deviation after a corrector replay).
int band_emit(mass_lb_handle* h, float* to, bool diag, cudaStream_t st)
{
  for(int i = 0; i < h->nbands; ++i)
  {
    const WallBand& b = h->band[i];
    const int nb = blocks_for(static_cast<long long>(b.map.BX)*b.map.BY);
    if(diag)
    {
      const State<float>& s = b.s;
      const BandDiag dd{{s.n, s.ux, s.uy, s.uxp, s.uyp, s.Hxx, s.Hyx, s.MU, s.dxQxx, s.dyQxx,
                         s.dxQyx, s.dyQyx, s.sXX, s.sYY, s.sYX, s.sXY, s.diag[0], s.diag[1],
                         s.diag[2], s.diag[3], s.diag[4], s.diag[5], s.diag[6]},
                        h->diag_n_dev ? 0.f : static_cast<float>(h->P.rho)};
      k_band_diag<<<nb, 256, 0, st>>>(b.map, h->diag, dd);
    }
    else k_band_scatter<<<nb, 256, 0, st>>>(b.map, to, band_ptrs(h, b));
    CU(cudaGetLastError(), "band scatter");
  }
  return 0;
}

// One fused step of a walled lattice: each band's work runs on its own
// high-priority stream beside the warp-strip kernel (both only read cur),
// then any further correctors (npc > 1), which reuse cur once the bands
// have read it; the step stream writes the band rows into the result,
// which is in nxt at the end.
int fused_step_with_bands(mass_lb_handle* h)
{
  CU(cudaEventRecord(h->band_in, h->stream), "band fork");
  for(int i = 0; i < h->nbands; ++i)
  {
    CU(cudaStreamWaitEvent(h->bstream[i], h->band_in, 0), "band fork");
    if(int r = band_compute(h, i, h->cur, h->bstream[i])) return r;
    CU(cudaEventRecord(h->band_out[i], h->bstream[i]), "band join");
  }
  const FusedArgs a = fused_args(h, h->cur, h->nxt, false);
  CU(launch_fused_step(a, h->model, h->cfg, false, h->stream), "fused step");
  for(unsigned c = 2; c <= h->P.npc; ++c)
  {
    if(c == 2)
      for(int i = 0; i < h->nbands; ++i)
        CU(cudaStreamWaitEvent(h->stream, h->band_read[i], 0), "band gather");
    if(int r = extra_corrector(h, h->nxt, h->cur, false)) return r;
    std::swap(h->cur, h->nxt);
  }
  for(int i = 0; i < h->nbands; ++i)
    CU(cudaStreamWaitEvent(h->stream, h->band_out[i], 0), "band join");
  return band_emit(h, h->nxt, false, h->stream);
}

int check_err_flag(mass_lb_handle* h)
{
  int e = 0;
  CU(cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "err flag");
  CU(cudaStreamSynchronize(h->stream), "sync");
  if(e) return fail(MASS_LB_ECUDA, "fused step: a bounded wait on a bulk copy timed out");
  return 0;
}

// Candidate tiles for the autotuner: strip widths that fit the lattice and
// chunk heights from 32 rows to the whole lattice, and from 2 rows on
// lattices of up to 2 M sites.
std::vector<FusedConfig> tile_candidates(const mass_lb_handle* h)
{
  std::vector<FusedConfig> c;
  for(int nt : {32, 64, 128, 256})
  {
    if(!fused_supported(static_cast<int>(h->LX), static_cast<int>(h->LY), nt)) continue;
    if(warp_strip_only(h) && nt != 32) continue;
    // 2 to 12 rows: on a small lattice the best chunk is the shortest whose
    // warps still fit in one wave (500^2: 4 rows, 282 CTAs)
    for(int rows : {2, 4, 6, 8, 12, 16, 32, 64, 128, 256, 512, 1024})
    {
      if(rows > static_cast<int>(h->LX) && rows != 8) continue;
      // short chunks only where a lattice has few strips to spread: each
      // warp's rows are a serial chain, and on a lattice whose state fits
      // in L2 more, shorter chains win over the pipeline fill they repeat
      if(rows < 32 && h->LX >= 32 && static_cast<long long>(h->LX)*h->LY > (1ll << 21)) continue;
      c.push_back(FusedConfig{nt, std::min(rows, static_cast<int>(h->LX))});
    }
  }
  return c;
}

int autotune(mass_lb_handle* h)
{
  const auto cands = tile_candidates(h);
  if(cands.empty()) return fail(MASS_LB_EUNSUPPORTED, "no fused tile fits this lattice");
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0), "event");
  CU(cudaEventCreate(&e1), "event");
  float best = 1e30f;
  FusedConfig bestc = cands.front();
  // time cur -> nxt without swapping: the state is not advanced
  for(const FusedConfig& c : cands)
  {
    const FusedArgs a = fused_args(h, h->cur, h->nxt, false);
    if(launch_fused_step(a, h->model, c, false, h->stream) != cudaSuccess) continue;
    CU(cudaEventRecord(e0, h->stream), "event");
    const int reps = 3;
    for(int r = 0; r < reps; ++r) launch_fused_step(a, h->model, c, false, h->stream);
    CU(cudaEventRecord(e1, h->stream), "event");
    CU(cudaEventSynchronize(e1), "event sync");
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, e0, e1), "event time");
    if(std::getenv("MASS_LB_TUNE_LOG"))
      std::fprintf(stderr, "mass_lb autotune: threads %d rows %d: %.4f ms/step\n",
                   c.nt, c.rows, ms/reps);
    if(ms < best) { best = ms; bestc = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->cfg = bestc;
  h->tuned = true;
  h->has_prev = false;   // nxt was used as scratch
  if(int r = check_err_flag(h)) return r;
  return 0;
}

int ensure_diag_buffer(mass_lb_handle* h)
{
  if(h->diag) return 0;
  return dalloc(h, &h->diag, static_cast<size_t>(NDIAG)*h->LX*h->LY);
}

} // namespace

// ==========================================================================

void mlb_set_last_error(const std::string& msg) { g_err = msg; }

extern "C" {

int mass_lb_abi_version(void) { return MASS_LB_ABI_VERSION; }

const char* mass_lb_last_error(void) { return g_err.c_str(); }

const char* mass_lb_field_name(int field)
{
  if(field < 0 || field >= MASS_LB_NUM_FIELDS) return nullptr;
  return kFieldNames[field];
}

int mass_lb_create(const mass_lb_params* params, unsigned LX, unsigned LY,
                   unsigned bc, int precision, mass_lb_handle** out)
{
  if(!params || !out) return fail(MASS_LB_EINVAL, "null argument");
  *out = nullptr;
  if(LX == 0 || LY == 0) return fail(MASS_LB_EINVAL, "empty lattice");
  if(params->model != MASS_LB_LYOTROPIC && params->model != MASS_LB_NEMATIC &&
     params->model != MASS_LB_GO_OR_GROW)
    return fail(MASS_LB_EINVAL, "unknown model");
  if(precision != MASS_LB_FP64 && precision != MASS_LB_FP32)
    return fail(MASS_LB_EINVAL, "unknown precision");
  if(params->npc < 1) return fail(MASS_LB_EINVAL, "npc must be >= 1");
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
  {
    cudaGetLastError();
    return fail(MASS_LB_ENODEV, "no CUDA device");
  }
  int dev = 0;
  CU(cudaGetDevice(&dev), "cudaGetDevice");
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
  if(prop.major != 10)
    return fail(MASS_LB_ENODEV, "this library is built for sm_100a (B200) only");

  auto* h = new mass_lb_handle();
  h->device = dev;
  h->precision = precision;
  h->model = params->model;
  h->LX = LX; h->LY = LY;
  h->bc = bc;
  // Which bc values carry walls: lyotropic and go-or-grow 1..4
  // (src/models/lyotropic.cpp:388-498, src/models/go-or-grow.cpp:393-418),
  // nematic 1 (src/models/nematic.cpp:259-368). Every other non-zero value is
  // the periodic ghost layer, which computes exactly what bc = 0 computes.
  h->wall = (h->model != NEM) ? (bc >= 1 && bc <= 4) : (bc == 1);
  if(h->wall && (LX < 2 || LY < 2))
  {
    delete h;
    return fail(MASS_LB_EINVAL, "wall boundaries need LX, LY >= 2");
  }
  std::memcpy(&h->P, params, sizeof(Params));
  static_assert(sizeof(Params) == sizeof(mass_lb_params), "param layout");
  const int g = h->wall ? 1 : 0;
  h->d = Dims{static_cast<int>(LX), static_cast<int>(LY), g,
              static_cast<int>(LX) + 2*g, static_cast<int>(LY) + 2*g,
              static_cast<long long>(LX + 2*g)*(LY + 2*g)};

  auto bail = [&](int r) { mass_lb_destroy(h); return r; };
  if(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MASS_LB_ECUDA, "stream create"));
  h->io = h->stream;
  {
    int least = 0, greatest = 0;
    if(cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
       cudaStreamCreateWithPriority(&h->xfer, cudaStreamNonBlocking, greatest) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->xfer_in, cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->xfer_out, cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->order_ev, cudaEventDisableTiming) != cudaSuccess)
      return bail(fail(MASS_LB_ECUDA, "transfer stream create"));
  }

  if(int r = dalloc(h, &h->err, 1)) return bail(r);
  if(int r = dalloc(h, &h->red_scratch, sums_scratch_doubles())) return bail(r);
  if(int r = dalloc(h, &h->red_out, 3)) return bail(r);
  const long long stage_sites = std::min<long long>(kStageSites, static_cast<long long>(LX)*LY);
  if(int r = dalloc(h, &h->stage, 9*stage_sites)) return bail(r);

  // go-or-grow defaults: the reference's initialisers (src/models/go-or-grow.hpp:11-13)
  // and phi_critical = 1
  const Pheno ph0{0., 1., 0., 0., 0., 0., 1., 0};
  h->s64.ph = ph0;
  h->s32.ph = ph0;
  if(precision == MASS_LB_FP64)
  {
    if(int r = alloc_state(h, h->s64)) return bail(r);
    if(int r = zero_state(h, h->s64)) return bail(r);
  }
  else
  {
    // the fused warp-strip kernel: every model with npc = 1 and lyotropic
    // and nematic lattices with npc > 1, periodic or, with the wall bands
    // beside it, walled; go-or-grow with npc > 1 runs the unfused sweeps
    h->fused = (h->P.npc == 1 || h->model != GOG) && (!h->wall || bands_fit(h)) &&
               fused_supported(static_cast<int>(LX), static_cast<int>(LY), 64);
    if(h->fused)
    {
      const size_t n = static_cast<size_t>(nplanes(h))*LX*LY;
      if(int r = dalloc(h, &h->cur, n)) return bail(r);
      if(int r = dalloc(h, &h->nxt, n)) return bail(r);
      if(cudaMemsetAsync(h->cur, 0, n*sizeof(float), h->stream) != cudaSuccess ||
         cudaMemsetAsync(h->nxt, 0, n*sizeof(float), h->stream) != cudaSuccess)
        return bail(fail(MASS_LB_ECUDA, "memset"));
      if(h->wall)
        if(int r = init_bands(h)) return bail(r);
      if(h->P.npc > 1)
      {
        const size_t np = static_cast<size_t>(h->model == NEM ? 11 : 12)*LX*LY;
        if(int r = dalloc(h, &h->pred, np)) return bail(r);
      }
      if(h->model == GOG)
      {
        // the growth-rate plane every go-or-grow step reads, zero until set
        const size_t np = static_cast<size_t>(LX)*LY;
        if(int r = dalloc(h, &h->src_fused, np)) return bail(r);
        if(cudaMemsetAsync(h->src_fused, 0, np*sizeof(float), h->stream) != cudaSuccess)
          return bail(fail(MASS_LB_ECUDA, "memset"));
      }
      if(const char* env = std::getenv("MASS_LB_TILE"))
      {
        int nt = 0, rows = 0;
        if(std::sscanf(env, "%d,%d", &nt, &rows) == 2 &&
           fused_supported(static_cast<int>(LX), static_cast<int>(LY), nt) && rows > 0 &&
           (nt == 32 || !warp_strip_only(h)))
        {
          h->cfg = FusedConfig{nt, rows};
          h->tuned = true;
        }
      }
      if(!h->tuned)
      {
        // the warp-strip kernel fits every fusable lattice; the autotuner
        // refines the tile on the first step
        h->cfg = FusedConfig{32, static_cast<int>(std::min(LX, 128u))};
      }
    }
    else
    {
      if(int r = alloc_state(h, h->s32)) return bail(r);
      if(int r = zero_state(h, h->s32)) return bail(r);
    }
  }
  if(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream) != cudaSuccess ||
     cudaStreamSynchronize(h->stream) != cudaSuccess)
    return bail(fail(MASS_LB_ECUDA, "init"));
  *out = h;
  return MASS_LB_OK;
}

void mass_lb_destroy(mass_lb_handle* h)
{
  if(!h) return;
  DeviceGuard g(h->device);
  if(h->stream) cudaStreamSynchronize(h->stream);
  for(void* p : h->allocs) cudaFree(p);
  if(h->mk_pinned) cudaFreeHost(h->mk_pinned);
  if(h->mk_copied) cudaEventDestroy(h->mk_copied);
  for(int i = 0; i < mass_lb_handle::MQ_STAGES; ++i)
  {
    if(h->mq_pinned[i]) cudaFreeHost(h->mq_pinned[i]);
    if(h->mq_copied[i]) cudaEventDestroy(h->mq_copied[i]);
  }
  for(int i = 0; i < mass_lb_handle::MQ_SLOTS; ++i)
  {
    if(h->mq_counted[i]) cudaEventDestroy(h->mq_counted[i]);
    if(h->mq_drew[i]) cudaEventDestroy(h->mq_drew[i]);
  }
  if(h->mq_host) cudaFreeHost(h->mq_host);
  if(h->tot_host) cudaFreeHost(h->tot_host);
  if(h->tot_ev) cudaEventDestroy(h->tot_ev);
  if(h->mq_copy) cudaStreamDestroy(h->mq_copy);
  if(h->xfer) { cudaStreamSynchronize(h->xfer); cudaStreamDestroy(h->xfer); }
  for(int i = 0; i < 2; ++i)
  {
    if(h->bstream[i]) { cudaStreamSynchronize(h->bstream[i]); cudaStreamDestroy(h->bstream[i]); }
    if(h->band_out[i]) cudaEventDestroy(h->band_out[i]);
    if(h->band_read[i]) cudaEventDestroy(h->band_read[i]);
  }
  if(h->band_in) cudaEventDestroy(h->band_in);
  if(h->xfer_in) cudaEventDestroy(h->xfer_in);
  if(h->xfer_out) cudaEventDestroy(h->xfer_out);
  if(h->order_ev) cudaEventDestroy(h->order_ev);
  if(h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

namespace {
cudaError_t launch_sums(mass_lb_handle* h);
int resolve_totals(mass_lb_handle* h);
bool pinned_host(const void* p);
} // namespace

// The derived fields of the last step, computed now if the step left them
// (before anything changes the state they come from, or when asked for).
static int settle_derived(mass_lb_handle* h)
{
  if(!h->derived_pending) return 0;
  h->derived_pending = false;
  const int r = h->precision == MASS_LB_FP64
    ? replay_derived_f64(h->d, h->P, h->s64, h->stream)
    : replay_derived_f32(h->d, h->P, h->s32, h->stream);
  if(r) return cuda_fail(cudaGetLastError(), "derived fields");
  return 0;
}

// One field transfer on the handle's high-priority transfer stream: it
// starts after the work queued on the step stream before it, and the step
// stream waits for it, so the order the caller sees on the handle's stream
// is unchanged. Only the conversion kernels and copies move; what follows
// the transfer is queued on the step stream again.
struct XferScope
{
  mass_lb_handle* h;
  explicit XferScope(mass_lb_handle* hh) : h(hh)
  {
    if(cudaEventRecord(h->xfer_in, h->stream) == cudaSuccess &&
       cudaStreamWaitEvent(h->xfer, h->xfer_in, 0) == cudaSuccess)
      h->io = h->xfer;
  }
  ~XferScope()
  {
    if(h->io == h->xfer)
    {
      cudaEventRecord(h->xfer_out, h->xfer);
      cudaStreamWaitEvent(h->stream, h->xfer_out, 0);
    }
    h->io = h->stream;
  }
  XferScope(const XferScope&) = delete;
  XferScope& operator=(const XferScope&) = delete;
};

// ff_raw: FP32 populations given as the deviations from t_v*rho the FP32
// state holds (a checkpoint's exact values), not as populations
static int put_field(mass_lb_handle* h, int field, const double* src, bool ff_raw = false)
{
  const int LY = static_cast<int>(h->LY);
  const long long rows_per = std::max<long long>(1, kStageSites/LY);
  const bool f64 = h->precision == MASS_LB_FP64;
  const bool isff = field == MASS_LB_FF;
  const int comps = isff ? 9 : 1;
  const double rest = f64 || ff_raw ? 0.0 : h->P.rho;
  {
  XferScope scope(h);   // joined before the chi update below
  for(long long x0 = 0; x0 < h->LX; x0 += rows_per)
  {
    const int nrows = static_cast<int>(std::min<long long>(rows_per, h->LX - x0));
    const long long n = static_cast<long long>(nrows)*LY;
    CU(cudaMemcpyAsync(h->stage, src + x0*LY*comps, n*comps*sizeof(double),
                       cudaMemcpyHostToDevice, h->io), "upload copy");
    const int nb = blocks_for(n);
    if(h->fused)
    {
      const long long plane = static_cast<long long>(h->LX)*h->LY;
      float* base = h->cur;
      if(isff)
        k_put_ff<float><<<nb, 256, 0, h->io>>>(h->stage, base, plane, x0, nrows, LY, 0, LY, rest);
      else
      {
        const int p = field == MASS_LB_QQXX ? 9 : field == MASS_LB_QQYX ? 10
                    : field == MASS_LB_M ? 12 : 11;
        k_put_scalar<float><<<nb, 256, 0, h->io>>>(h->stage, base + p*plane, x0, nrows, LY, 0, LY);
      }
    }
    else if(f64)
    {
      State<double>& s = h->s64;
      double* a = field == MASS_LB_QQXX ? s.Qxx : field == MASS_LB_QQYX ? s.Qyx
                : field == MASS_LB_M ? s.m : s.phi;
      if(isff) k_put_ff<double><<<nb, 256, 0, h->io>>>(h->stage, s.ff, h->d.NE, x0, nrows, LY, h->d.g, h->d.EY, 0.0);
      else k_put_scalar<double><<<nb, 256, 0, h->io>>>(h->stage, a, x0, nrows, LY, h->d.g, h->d.EY);
    }
    else
    {
      State<float>& s = h->s32;
      float* a = field == MASS_LB_QQXX ? s.Qxx : field == MASS_LB_QQYX ? s.Qyx
               : field == MASS_LB_M ? s.m : s.phi;
      if(isff) k_put_ff<float><<<nb, 256, 0, h->io>>>(h->stage, s.ff, h->d.NE, x0, nrows, LY, h->d.g, h->d.EY, rest);
      else k_put_scalar<float><<<nb, 256, 0, h->io>>>(h->stage, a, x0, nrows, LY, h->d.g, h->d.EY);
    }
    CU(cudaGetLastError(), "upload kernel");
  }
  }
  // chi follows phi and m (the fused kernel forms chi = m/phi itself)
  if(h->model == GOG && !h->fused && (field == MASS_LB_PHI || field == MASS_LB_M))
  {
    const int r = h->precision == MASS_LB_FP64 ? update_chi_f64(h->d, h->s64, h->stream)
                                               : update_chi_f32(h->d, h->s32, h->stream);
    if(r) return cuda_fail(cudaGetLastError(), "chi update");
  }
  return 0;
}

int mass_lb_upload_field(mass_lb_handle* h, int field, const double* src)
{
  if(!h || !src) return fail(MASS_LB_EINVAL, "null argument");
  if(field != MASS_LB_FF && field != MASS_LB_QQXX && field != MASS_LB_QQYX &&
     field != MASS_LB_PHI && field != MASS_LB_M)
    return fail(MASS_LB_EINVAL, "only ff, QQxx, QQyx, phi and m can be uploaded");
  if(field == MASS_LB_PHI && h->model == NEM)
    return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  if(field == MASS_LB_M && h->model != GOG)
    return fail(MASS_LB_EUNSUPPORTED, "m exists in the go-or-grow model only");
  DeviceGuard g(h->device);
  if(int r = settle_derived(h)) return r;
  if(int r = put_field(h, field, src)) return r;
  h->has_prev = false;
  CU(cudaStreamSynchronize(h->stream), "upload sync");
  return 0;
}

static int upload_state(mass_lb_handle* h, const double* ff, const double* QQxx,
                        const double* QQyx, const double* phi, bool ff_raw);

int mass_lb_upload(mass_lb_handle* h, const double* ff, const double* QQxx,
                   const double* QQyx, const double* phi)
{
  return upload_state(h, ff, QQxx, QQyx, phi, false);
}

static int upload_state(mass_lb_handle* h, const double* ff, const double* QQxx,
                        const double* QQyx, const double* phi, bool ff_raw)
{
  if(!h || !ff || !QQxx || !QQyx) return fail(MASS_LB_EINVAL, "null argument");
  if(h->model != NEM && !phi) return fail(MASS_LB_EINVAL, "lyotropic models need phi");
  DeviceGuard g(h->device);
  if(int r = settle_derived(h)) return r;
  if(int r = put_field(h, MASS_LB_FF, ff, ff_raw)) return r;
  if(int r = put_field(h, MASS_LB_QQXX, QQxx)) return r;
  if(int r = put_field(h, MASS_LB_QQYX, QQyx)) return r;
  if(h->model != NEM)
    if(int r = put_field(h, MASS_LB_PHI, phi)) return r;
  h->has_prev = false;
  h->steps = 0;
  // reference totals (ftot, ptot), as Configure() accumulates them
  double fs = 0, ps = 0;
  int bad = 0;
  if(int r = mass_lb_checks(h, &fs, &ps, &bad)) return r;
  if(int r = resolve_totals(h)) return r;   // an earlier asynchronous upload's
  h->ftot = fs;
  h->ptot = ps;
  return 0;
}

int mass_lb_upload_async(mass_lb_handle* h, const double* ff, const double* QQxx,
                         const double* QQyx, const double* phi)
{
  if(!h || !ff || !QQxx || !QQyx) return fail(MASS_LB_EINVAL, "null argument");
  if(h->model != NEM && !phi) return fail(MASS_LB_EINVAL, "lyotropic models need phi");
  DeviceGuard g(h->device);
  if(!pinned_host(ff) || !pinned_host(QQxx) || !pinned_host(QQyx) ||
     (h->model != NEM && !pinned_host(phi)))
    return fail(MASS_LB_EINVAL, "asynchronous uploads take pinned host buffers");
  if(int r = settle_derived(h)) return r;
  if(int r = resolve_totals(h)) return r;
  if(!h->tot_host)
  {
    CU(cudaMallocHost(reinterpret_cast<void**>(&h->tot_host), 3*sizeof(double)), "pinned");
    CU(cudaEventCreateWithFlags(&h->tot_ev, cudaEventDisableTiming), "event");
  }
  if(int r = put_field(h, MASS_LB_FF, ff)) return r;
  if(int r = put_field(h, MASS_LB_QQXX, QQxx)) return r;
  if(int r = put_field(h, MASS_LB_QQYX, QQyx)) return r;
  if(h->model != NEM)
    if(int r = put_field(h, MASS_LB_PHI, phi)) return r;
  h->has_prev = false;
  h->steps = 0;
  // the reference totals follow on the stream; read when first asked for
  const cudaError_t e = launch_sums(h);
  if(e != cudaSuccess) return cuda_fail(e, "sums");
  CU(cudaMemcpyAsync(h->tot_host, h->red_out, 3*sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream), "sums copy");
  CU(cudaEventRecord(h->tot_ev, h->stream), "event");
  h->tot_pending = true;
  return 0;
}

int mass_lb_step(mass_lb_handle* h, unsigned nsteps)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(nsteps == 0) return 0;
  DeviceGuard g(h->device);
  const int bc = h->wall ? static_cast<int>(h->bc) : 0;
  // sub-step kernels leave the derived fields to a replay on demand
  const bool lazy = !h->fused && substep_path(h->d, h->P, bc);
  if(h->precision == MASS_LB_FP64)
  {
    if(step_unfused_f64(h->d, h->P, h->s64, bc, nsteps, !lazy, h->stream) != 0)
      return cuda_fail(cudaGetLastError(), "fp64 step");
    h->derived_pending = lazy;
  }
  else if(!h->fused)
  {
    if(step_unfused_f32(h->d, h->P, h->s32, bc, nsteps, !lazy, h->stream) != 0)
      return cuda_fail(cudaGetLastError(), "fp32 step");
    h->derived_pending = lazy;
  }
  else
  {
    if(!h->tuned)
      if(int r = autotune(h)) return r;
    for(unsigned i = 0; i < nsteps; ++i)
    {
      if(h->nbands)
      {
        if(int r = fused_step_with_bands(h)) return r;
      }
      else
      {
        const FusedArgs a = fused_args(h, h->cur, h->nxt, false);
        CU(launch_fused_step(a, h->model, h->cfg, false, h->stream), "fused step");
        // npc > 1: the further correctors; the last one's input stays in
        // nxt after the swap below, for the derived-field replay
        for(unsigned c = 2; c <= h->P.npc; ++c)
        {
          if(int r = extra_corrector(h, h->nxt, h->cur, false)) return r;
          std::swap(h->cur, h->nxt);
        }
      }
      std::swap(h->cur, h->nxt);
    }
    h->has_prev = true;
  }
  h->steps += nsteps;
  return 0;
}

// ff_raw: FP32 populations as the stored deviations from t_v*rho
static int get_primary(mass_lb_handle* h, int field, double* out, bool sync = true,
                       bool ff_raw = false)
{
  const double rest32 = ff_raw ? 0.0 : h->P.rho;
  const int LY = static_cast<int>(h->LY);
  const long long rows_per = std::max<long long>(1, kStageSites/LY);
  const bool isff = field == MASS_LB_FF || field == MASS_LB_FN;
  const int comps = isff ? 9 : 1;
  {
  XferScope scope(h);
  for(long long x0 = 0; x0 < h->LX; x0 += rows_per)
  {
    const int nrows = static_cast<int>(std::min<long long>(rows_per, h->LX - x0));
    const long long n = static_cast<long long>(nrows)*LY;
    const int nb = blocks_for(n);
    if(h->fused)
    {
      const long long plane = static_cast<long long>(h->LX)*h->LY;
      if(field == MASS_LB_M)
        k_get_scalar<float><<<nb, 256, 0, h->io>>>(h->stage, h->cur + 12*plane, x0, nrows, LY, 0, LY, 0.0);
      else if(field == MASS_LB_CHI)
        k_get_chi<<<nb, 256, 0, h->io>>>(h->stage, h->cur + 11*plane, h->cur + 12*plane,
                                             x0, nrows, LY);
      else if(field <= MASS_LB_PHI)
      {
        if(isff) k_get_ff<float><<<nb, 256, 0, h->io>>>(h->stage, h->cur, plane, x0, nrows, LY, 0, LY, rest32);
        else
        {
          const int p = field == MASS_LB_QQXX ? 9 : field == MASS_LB_QQYX ? 10 : 11;
          k_get_scalar<float><<<nb, 256, 0, h->io>>>(h->stage, h->cur + p*plane, x0, nrows, LY, 0, LY, 0.0);
        }
      }
      else
      {
        // derived fields from the replayed diagnostics, mass_lb_field order
        const int p = field - MASS_LB_N;
        k_get_scalar<float><<<nb, 256, 0, h->io>>>(h->stage, h->diag + p*plane, x0, nrows, LY, 0, LY,
                                                   p == 0 && h->diag_n_dev ? h->P.rho : 0.0);
      }
    }
    else if(h->precision == MASS_LB_FP64)
    {
      State<double>& s = h->s64;
      const Dims& d = h->d;
      const double* a = nullptr;
      switch(field)
      {
        case MASS_LB_QQXX: a = s.Qxx; break;  case MASS_LB_QQYX: a = s.Qyx; break;
        case MASS_LB_PHI: a = s.phi; break;   case MASS_LB_N: a = s.n; break;
        case MASS_LB_UX: a = s.ux; break;     case MASS_LB_UY: a = s.uy; break;
        case MASS_LB_UX_PHI: a = s.uxp; break; case MASS_LB_UY_PHI: a = s.uyp; break;
        case MASS_LB_HHXX: a = s.Hxx; break;  case MASS_LB_HHYX: a = s.Hyx; break;
        case MASS_LB_MU: a = s.MU; break;
        case MASS_LB_DXQQXX: a = s.dxQxx; break; case MASS_LB_DYQQXX: a = s.dyQxx; break;
        case MASS_LB_DXQQYX: a = s.dxQyx; break; case MASS_LB_DYQQYX: a = s.dyQyx; break;
        case MASS_LB_SIGMAXX: a = s.sXX; break; case MASS_LB_SIGMAYY: a = s.sYY; break;
        case MASS_LB_SIGMAYX: a = s.sYX; break; case MASS_LB_SIGMAXY: a = s.sXY; break;
        case MASS_LB_QNXX: a = s.QNxx; break; case MASS_LB_QNYX: a = s.QNyx; break;
        case MASS_LB_PHN: a = s.phn; break;
        case MASS_LB_M: a = s.m; break;       case MASS_LB_CHI: a = s.chi; break;
        case MASS_LB_MN: a = s.mN; break;
        default:
          if(field >= MASS_LB_SIGMA_BULK && field <= MASS_LB_SIGMA_ACTIVE_YX)
            a = s.diag[field - MASS_LB_SIGMA_BULK];
      }
      if(field == MASS_LB_FF) k_get_ff<double><<<nb, 256, 0, h->io>>>(h->stage, s.ff, d.NE, x0, nrows, LY, d.g, d.EY, 0.0);
      else if(field == MASS_LB_FN) k_get_ff<double><<<nb, 256, 0, h->io>>>(h->stage, s.fn, d.NE, x0, nrows, LY, d.g, d.EY, 0.0);
      else k_get_scalar<double><<<nb, 256, 0, h->io>>>(h->stage, a, x0, nrows, LY, d.g, d.EY, 0.0);
    }
    else
    {
      State<float>& s = h->s32;
      const Dims& d = h->d;
      const float* a = nullptr;
      double add = 0.0;
      switch(field)
      {
        case MASS_LB_QQXX: a = s.Qxx; break;  case MASS_LB_QQYX: a = s.Qyx; break;
        case MASS_LB_PHI: a = s.phi; break;   case MASS_LB_N: a = s.n; add = h->P.rho; break;
        case MASS_LB_UX: a = s.ux; break;     case MASS_LB_UY: a = s.uy; break;
        case MASS_LB_UX_PHI: a = s.uxp; break; case MASS_LB_UY_PHI: a = s.uyp; break;
        case MASS_LB_HHXX: a = s.Hxx; break;  case MASS_LB_HHYX: a = s.Hyx; break;
        case MASS_LB_MU: a = s.MU; break;
        case MASS_LB_DXQQXX: a = s.dxQxx; break; case MASS_LB_DYQQXX: a = s.dyQxx; break;
        case MASS_LB_DXQQYX: a = s.dxQyx; break; case MASS_LB_DYQQYX: a = s.dyQyx; break;
        case MASS_LB_SIGMAXX: a = s.sXX; break; case MASS_LB_SIGMAYY: a = s.sYY; break;
        case MASS_LB_SIGMAYX: a = s.sYX; break; case MASS_LB_SIGMAXY: a = s.sXY; break;
        case MASS_LB_M: a = s.m; break;       case MASS_LB_CHI: a = s.chi; break;
        default:
          if(field >= MASS_LB_SIGMA_BULK && field <= MASS_LB_SIGMA_ACTIVE_YX)
            a = s.diag[field - MASS_LB_SIGMA_BULK];
      }
      if(field == MASS_LB_FF) k_get_ff<float><<<nb, 256, 0, h->io>>>(h->stage, s.ff, d.NE, x0, nrows, LY, d.g, d.EY, rest32);
      else k_get_scalar<float><<<nb, 256, 0, h->io>>>(h->stage, a, x0, nrows, LY, d.g, d.EY, add);
    }
    CU(cudaGetLastError(), "download kernel");
    CU(cudaMemcpyAsync(out + x0*LY*comps, h->stage, n*comps*sizeof(double),
                       cudaMemcpyDeviceToHost, h->io), "download copy");
  }
  }
  if(sync) CU(cudaStreamSynchronize(h->stream), "download sync");
  return 0;
}

int mass_lb_download(mass_lb_handle* h, int field, double* out)
{
  if(!h || !out) return fail(MASS_LB_EINVAL, "null argument");
  if(field < 0 || field >= MASS_LB_NUM_FIELDS) return fail(MASS_LB_EINVAL, "bad field id");
  const bool phase_field = field == MASS_LB_PHI || field == MASS_LB_UX_PHI ||
    field == MASS_LB_UY_PHI || field == MASS_LB_MU || field == MASS_LB_PHN ||
    (field >= MASS_LB_SIGMA_BULK && field <= MASS_LB_SIGMA_ACTIVE_YX);
  if(h->model == NEM && phase_field)
    return fail(MASS_LB_EUNSUPPORTED, "field does not exist in the nematic model");
  if(h->model != GOG && (field == MASS_LB_M || field == MASS_LB_CHI || field == MASS_LB_MN))
    return fail(MASS_LB_EUNSUPPORTED, "m and chi exist in the go-or-grow model only");
  const bool predictor = (field >= MASS_LB_FN && field <= MASS_LB_PHN) || field == MASS_LB_MN;
  if(h->precision == MASS_LB_FP32 && predictor)
    return fail(MASS_LB_EUNSUPPORTED, "step-internal predictor fields are FP64-mode only");
  DeviceGuard g(h->device);
  if(!h->fused && field >= MASS_LB_N && field <= MASS_LB_SIGMA_ACTIVE_YX)
    if(int r = settle_derived(h)) return r;
  if(h->fused && field >= MASS_LB_N && field <= MASS_LB_SIGMA_ACTIVE_YX)
  {
    if(!h->has_prev)
      return fail(MASS_LB_EUNSUPPORTED, "derived fields need a step since the last upload");
    if(int r = ensure_diag_buffer(h)) return r;
    if(h->P.npc > 1)
    {
      // the last corrector again, from its input (nxt) and the step's
      // predictor values, its outputs thrown away
      if(!h->scratch)
        if(int r = dalloc(h, &h->scratch, static_cast<size_t>(nplanes(h))*h->LX*h->LY)) return r;
      if(int r = extra_corrector(h, h->nxt, h->scratch, true)) return r;
      h->diag_n_dev = true;
    }
    else
    {
      // replay the last step from the retained input with the diagnostic
      // outputs on (the replay does not write the state)
      const FusedArgs a = fused_args(h, h->nxt, h->cur, true);
      CU(launch_fused_step(a, h->model, h->cfg, true, h->stream), "diag replay");
      h->diag_n_dev = false;
    }
    // the wall bands kept theirs when they stepped
    if(h->nbands)
      if(int r = band_emit(h, nullptr, true, h->stream)) return r;
    if(int r = check_err_flag(h)) return r;
  }
  return get_primary(h, field, out);
}

int mass_lb_download_async(mass_lb_handle* h, int field, double* out)
{
  if(!h || !out) return fail(MASS_LB_EINVAL, "null argument");
  if(field != MASS_LB_FF && field != MASS_LB_QQXX && field != MASS_LB_QQYX &&
     field != MASS_LB_PHI)
    return fail(MASS_LB_EINVAL, "asynchronous downloads take ff, QQxx, QQyx or phi");
  if(field == MASS_LB_PHI && h->model == NEM)
    return fail(MASS_LB_EUNSUPPORTED, "field does not exist in the nematic model");
  DeviceGuard g(h->device);
  if(!pinned_host(out))
    return fail(MASS_LB_EINVAL, "asynchronous downloads take pinned host buffers");
  return get_primary(h, field, out, false);
}

} // extern "C"

namespace {

// Sum of f and phi and the non-finite count into red_out (3 doubles), on
// the handle's stream.
cudaError_t launch_sums(mass_lb_handle* h)
{
  cudaError_t e;
  if(h->fused)
  {
    const long long plane = static_cast<long long>(h->LX)*h->LY;
    SumView<float> v{h->cur, h->cur + 9*plane, h->cur + 10*plane,
                     h->model != NEM ? h->cur + 11*plane : nullptr, plane,
                     static_cast<int>(h->LX), static_cast<int>(h->LY), 0,
                     static_cast<int>(h->LY), h->P.rho};
    e = launch_sums_f32(v, h->red_scratch, h->red_out, h->stream);
  }
  else if(h->precision == MASS_LB_FP64)
  {
    const State<double>& s = h->s64;
    SumView<double> v{s.ff, s.Qxx, s.Qyx, h->model != NEM ? s.phi : nullptr, h->d.NE,
                      h->d.LX, h->d.LY, h->d.g, h->d.EY, 0.0};
    e = launch_sums_f64(v, h->red_scratch, h->red_out, h->stream);
  }
  else
  {
    const State<float>& s = h->s32;
    SumView<float> v{s.ff, s.Qxx, s.Qyx, h->model != NEM ? s.phi : nullptr, h->d.NE,
                     h->d.LX, h->d.LY, h->d.g, h->d.EY, h->P.rho};
    e = launch_sums_f32(v, h->red_scratch, h->red_out, h->stream);
  }
  return e;
}

// ftot/ptot of an asynchronous upload, once its sums have landed
int resolve_totals(mass_lb_handle* h)
{
  if(!h->tot_pending) return 0;
  CU(cudaEventSynchronize(h->tot_ev), "totals");
  h->ftot = h->tot_host[0];
  h->ptot = h->tot_host[1];
  h->tot_pending = false;
  return 0;
}

bool pinned_host(const void* p)
{
  cudaPointerAttributes a{};
  if(cudaPointerGetAttributes(&a, p) != cudaSuccess)
  {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// ---- rows of the primary state (domain decomposition) ---------------------

// Base pointer and plane geometry of primary plane q (0..8 populations, 9
// Qxx, 10 Qyx, 11 phi) in the handle's own storage: element pointer of row
// 0, column 0, and the row pitch in elements.
template<typename T>
T* primary_plane(mass_lb_handle* h, State<T>& s, int q, long long* pitch)
{
  *pitch = h->d.EY;
  const long long off = static_cast<long long>(h->d.EY)*h->d.g + h->d.g;
  T* base = q < 9 ? s.ff + q*h->d.NE : q == 9 ? s.Qxx : q == 10 ? s.Qyx : s.phi;
  return base + off;
}

// Row r of plane q of the state, for r in [0, nrows): p[q] + r*pitch + y.
template<typename T>
struct RowPlanes
{
  T* p[13];
};

// state rows <-> packed [plane][row][y], one thread per value
template<typename T>
__global__ void __launch_bounds__(256)
k_copy_rows(RowPlanes<T> pl, T* __restrict__ packed, int np, int nrows, int LY, long long pitch,
            int to_rows)
{
  const long long per = static_cast<long long>(nrows)*LY, total = per*np;
  for(long long k = blockIdx.x*256ll + threadIdx.x; k < total; k += 256ll*gridDim.x)
  {
    const int q = static_cast<int>(k / per);
    const long long rem = k - q*per;
    const long long r = rem / LY, y = rem - r*LY;
    T* st = pl.p[q] + r*pitch + y;
    if(to_rows) *st = packed[k];
    else packed[k] = *st;
  }
}

// Copies rows [x0, x0+nrows) of every primary plane between the handle's
// state and a packed device buffer laid out [plane][row][y]. `to_rows`
// selects the direction (packed -> state). One kernel launch on the
// handle's stream (strided copy-engine transfers of a few rows per plane
// cost more than the bytes they move).
int copy_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, void* packed, bool to_rows)
{
  if(!h || !packed) return fail(MASS_LB_EINVAL, "null argument");
  if(h->model == GOG)
    return fail(MASS_LB_EUNSUPPORTED, "row transfers cover the lyotropic and nematic models");
  if(h->wall) return fail(MASS_LB_EUNSUPPORTED, "row transfers need a periodic lattice");
  if(nrows == 0 || x0 >= h->LX || nrows > h->LX - x0)
    return fail(MASS_LB_EINVAL, "row range outside the lattice");
  DeviceGuard g(h->device);
  if(to_rows)
    if(int r = settle_derived(h)) return r;
  const int NP = nplanes(h);
  const int LY = static_cast<int>(h->LY);
  const long long total = static_cast<long long>(NP)*nrows*LY;
  const int nb = blocks_for(total);
  if(h->fused)
  {
    // planes of LX*LY floats
    RowPlanes<float> pl{};
    const long long plane = static_cast<long long>(h->LX)*LY;
    for(int q = 0; q < NP; ++q) pl.p[q] = h->cur + q*plane + static_cast<long long>(x0)*LY;
    k_copy_rows<float><<<nb, 256, 0, h->stream>>>(pl, static_cast<float*>(packed), NP,
                                                  static_cast<int>(nrows), LY, LY, to_rows);
    CU(cudaGetLastError(), "row copy");
    if(to_rows) h->has_prev = false;
    return 0;
  }
  long long pitch = 0;
  if(h->precision == MASS_LB_FP64)
  {
    RowPlanes<double> pl{};
    for(int q = 0; q < NP; ++q)
      pl.p[q] = primary_plane(h, h->s64, q, &pitch) + static_cast<long long>(x0)*pitch;
    k_copy_rows<double><<<nb, 256, 0, h->stream>>>(pl, static_cast<double*>(packed), NP,
                                                   static_cast<int>(nrows), LY, pitch, to_rows);
  }
  else
  {
    RowPlanes<float> pl{};
    for(int q = 0; q < NP; ++q)
      pl.p[q] = primary_plane(h, h->s32, q, &pitch) + static_cast<long long>(x0)*pitch;
    k_copy_rows<float><<<nb, 256, 0, h->stream>>>(pl, static_cast<float*>(packed), NP,
                                                  static_cast<int>(nrows), LY, pitch, to_rows);
  }
  CU(cudaGetLastError(), "row copy");
  return 0;
}

} // namespace

extern "C" {

int mass_lb_checks(mass_lb_handle* h, double* fsum, double* phisum, int* nonfinite)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  DeviceGuard g(h->device);
  const cudaError_t e = launch_sums(h);
  if(e != cudaSuccess) return cuda_fail(e, "sums");
  double r[3];
  CU(cudaMemcpyAsync(r, h->red_out, sizeof(r), cudaMemcpyDeviceToHost, h->stream), "sums copy");
  CU(cudaStreamSynchronize(h->stream), "sums sync");
  if(h->fused)
    if(int rc = check_err_flag(h)) return rc;
  if(fsum) *fsum = r[0];
  if(phisum) *phisum = r[1];
  if(nonfinite) *nonfinite = r[2] != 0.0 ? 1 : 0;
  return 0;
}

int mass_lb_rows_layout(mass_lb_handle* h, int* nplanes_out, int* elem_bytes)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(nplanes_out) *nplanes_out = nplanes(h);
  if(elem_bytes) *elem_bytes = h->precision == MASS_LB_FP64 ? 8 : 4;
  return 0;
}

int mass_lb_set_step_rows(mass_lb_handle* h, unsigned x0, unsigned nrows)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(nrows == 0) { h->step_x0 = h->step_nx = 0; return 0; }
  if(!h->fused || h->wall || h->P.npc != 1 || h->in_ensemble)
    return fail(MASS_LB_EUNSUPPORTED,
                "row-range steps need a fused periodic lattice with npc = 1");
  if(x0 >= h->LX || nrows > h->LX - x0)
    return fail(MASS_LB_EINVAL, "row range outside the lattice");
  h->step_x0 = x0;
  h->step_nx = nrows;
  h->has_prev = false;
  return 0;
}

int mass_lb_get_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, void* dst)
{
  return copy_rows(h, x0, nrows, dst, false);
}

int mass_lb_put_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, const void* src)
{
  return copy_rows(h, x0, nrows, const_cast<void*>(src), true);
}

int mass_lb_checks_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, double* fsum,
                        double* phisum, int* nonfinite)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(nrows == 0 || x0 >= h->LX || nrows > h->LX - x0)
    return fail(MASS_LB_EINVAL, "row range outside the lattice");
  DeviceGuard g(h->device);
  cudaError_t e;
  if(h->fused)
  {
    const long long plane = static_cast<long long>(h->LX)*h->LY;
    const float* b = h->cur + static_cast<long long>(x0)*h->LY;
    SumView<float> v{b, b + 9*plane, b + 10*plane, h->model != NEM ? b + 11*plane : nullptr,
                     plane, static_cast<int>(nrows), static_cast<int>(h->LY), 0,
                     static_cast<int>(h->LY), h->P.rho};
    e = launch_sums_f32(v, h->red_scratch, h->red_out, h->stream);
  }
  else if(h->precision == MASS_LB_FP64)
  {
    const State<double>& s = h->s64;
    const long long o = static_cast<long long>(h->d.EY)*x0;
    SumView<double> v{s.ff + o, s.Qxx + o, s.Qyx + o, h->model != NEM ? s.phi + o : nullptr,
                      h->d.NE, static_cast<int>(nrows), h->d.LY, h->d.g, h->d.EY, 0.0};
    e = launch_sums_f64(v, h->red_scratch, h->red_out, h->stream);
  }
  else
  {
    const State<float>& s = h->s32;
    const long long o = static_cast<long long>(h->d.EY)*x0;
    SumView<float> v{s.ff + o, s.Qxx + o, s.Qyx + o, h->model != NEM ? s.phi + o : nullptr,
                     h->d.NE, static_cast<int>(nrows), h->d.LY, h->d.g, h->d.EY, h->P.rho};
    e = launch_sums_f32(v, h->red_scratch, h->red_out, h->stream);
  }
  if(e != cudaSuccess) return cuda_fail(e, "sums");
  double r[3];
  CU(cudaMemcpyAsync(r, h->red_out, sizeof(r), cudaMemcpyDeviceToHost, h->stream), "sums copy");
  CU(cudaStreamSynchronize(h->stream), "sums sync");
  if(h->fused)
    if(int rc = check_err_flag(h)) return rc;
  if(fsum) *fsum = r[0];
  if(phisum) *phisum = r[1];
  if(nonfinite) *nonfinite = r[2] != 0.0 ? 1 : 0;
  return 0;
}

int mass_lb_initial_totals(mass_lb_handle* h, double* ftot, double* ptot)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  DeviceGuard g(h->device);
  if(int r = resolve_totals(h)) return r;
  if(ftot) *ftot = h->ftot;
  if(ptot) *ptot = h->ptot;
  return 0;
}

int mass_lb_synchronize(mass_lb_handle* h)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  DeviceGuard g(h->device);
  CU(cudaStreamSynchronize(h->stream), "sync");
  if(h->fused) return check_err_flag(h);
  return 0;
}

void* mass_lb_stream(mass_lb_handle* h) { return h ? static_cast<void*>(h->stream) : nullptr; }

int mass_lb_stream_wait(mass_lb_handle* h, mass_lb_handle* before)
{
  if(!h || !before) return fail(MASS_LB_EINVAL, "null handle");
  if(h == before) return 0;
  {
    DeviceGuard g(before->device);
    CU(cudaEventRecord(before->order_ev, before->stream), "order mark");
  }
  DeviceGuard g(h->device);
  CU(cudaStreamWaitEvent(h->stream, before->order_ev, 0), "order wait");
  return 0;
}

int mass_lb_launches_per_step(mass_lb_handle* h)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  // fused with walls: per band a gather, [chi,] the wall sweeps, a scatter
  // npc > 1: a corrector sub-step per further corrector
  if(h->fused)
    return static_cast<int>(h->P.npc) +
           h->nbands*(2 + (h->model == GOG ? 1 : 0) +
                      launches_unfused(h->model, static_cast<int>(h->bc), h->P.npc));
  return launches_unfused(h->model, h->wall ? static_cast<int>(h->bc) : 0, h->P.npc);
}

// ---- mass_lb_ext.h ------------------------------------------------------

int mass_lb_get_tile(mass_lb_handle* h, int* threads, int* rows)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(!h->fused) return fail(MASS_LB_EUNSUPPORTED, "not using the fused kernel");
  if(threads) *threads = h->cfg.nt;
  if(rows) *rows = h->cfg.rows;
  return 0;
}

int mass_lb_set_tile(mass_lb_handle* h, int threads, int rows)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(!h->fused) return fail(MASS_LB_EUNSUPPORTED, "not using the fused kernel");
  if(threads == 0 && rows == 0) { h->tuned = false; return 0; }
  if(!fused_supported(static_cast<int>(h->LX), static_cast<int>(h->LY), threads) || rows <= 0)
    return fail(MASS_LB_EINVAL, "tile does not fit this lattice");
  if(threads != 32 && warp_strip_only(h))
    return fail(MASS_LB_EUNSUPPORTED,
                "a phi source, go-or-grow and npc > 1 need the warp-strip kernel (threads = 32)");
  h->cfg = FusedConfig{threads, rows};
  h->tuned = true;
  return 0;
}

int mass_lb_autotune(mass_lb_handle* h)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(!h->fused) return 0;
  DeviceGuard g(h->device);
  return autotune(h);
}

int mass_lb_uses_fused(mass_lb_handle* h) { return h && h->fused ? 1 : 0; }

int mass_lb_statistics(mass_lb_handle* h, mass_lb_stats* out)
{
  if(!h || !out) return fail(MASS_LB_EINVAL, "null argument");
  DeviceGuard g(h->device);
  const long long N = static_cast<long long>(h->LX)*h->LY;
  if(!h->stats.U)
  {
    StatScratch& s = h->stats;
    if(int r = dalloc(h, &s.U, 2*N)) return r;
    if(int r = dalloc(h, &s.D, 2*N)) return r;
    if(int r = dalloc(h, &s.partial, 8*STATS_BLOCKS)) return r;
    if(int r = dalloc(h, &s.out, 5)) return r;
    if(int r = dalloc(h, &s.count, 1)) return r;
    if(int r = dalloc(h, &s.list, N)) return r;
    s.capacity = static_cast<int>(std::min<long long>(N, 0x7fffffff));
  }
  cudaError_t e;
  if(h->fused)
  {
    const long long plane = N;
    StatView<float> v{h->cur, plane, h->cur + 9*plane, h->cur + 10*plane,
                      h->model != NEM ? h->cur + 11*plane : nullptr,
                      static_cast<int>(h->LX), static_cast<int>(h->LY), 0,
                      static_cast<int>(h->LY), h->P.rho};
    e = launch_stats_f32(v, h->stats, 0.4, h->stream);
  }
  else if(h->precision == MASS_LB_FP64)
  {
    const State<double>& s = h->s64;
    StatView<double> v{s.ff, h->d.NE, s.Qxx, s.Qyx, h->model != NEM ? s.phi : nullptr,
                       h->d.LX, h->d.LY, h->d.g, h->d.EY, 0.0};
    e = launch_stats_f64(v, h->stats, 0.4, h->stream);
  }
  else
  {
    const State<float>& s = h->s32;
    StatView<float> v{s.ff, h->d.NE, s.Qxx, s.Qyx, h->model != NEM ? s.phi : nullptr,
                      h->d.LX, h->d.LY, h->d.g, h->d.EY, h->P.rho};
    e = launch_stats_f32(v, h->stats, 0.4, h->stream);
  }
  if(e != cudaSuccess) return cuda_fail(e, "statistics");
  double sums[5];
  int count = 0;
  CU(cudaMemcpyAsync(sums, h->stats.out, sizeof(sums), cudaMemcpyDeviceToHost, h->stream), "stats copy");
  CU(cudaMemcpyAsync(&count, h->stats.count, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "stats copy");
  CU(cudaStreamSynchronize(h->stream), "stats sync");
  if(count > h->stats.capacity) return fail(MASS_LB_ECUDA, "charged-site list overflow");
  std::vector<int> list(count);
  if(count)
  {
    CU(cudaMemcpy(list.data(), h->stats.list, count*sizeof(int), cudaMemcpyDeviceToHost), "stats list");
  }
  // Cluster the charged sites: 4-connected (periodic) same-sign components,
  // one defect each, as the breadth-first search of defects.py:75-95.
  std::sort(list.begin(), list.end());
  std::vector<int> parent(count);
  for(int i = 0; i < count; ++i) parent[i] = i;
  auto find = [&](int i) {
    while(parent[i] != i) { parent[i] = parent[parent[i]]; i = parent[i]; }
    return i;
  };
  const int LX = static_cast<int>(h->LX), LY = static_cast<int>(h->LY);
  for(int i = 0; i < count; ++i)
  {
    const int code = list[i];
    const bool plus = code >= 0;
    const long long k = plus ? code : -static_cast<long long>(code) - 1;
    const int x = static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    const int nx[4] = {(x + 1) % LX, (x + LX - 1) % LX, x, x};
    const int ny[4] = {y, y, (y + 1) % LY, (y + LY - 1) % LY};
    for(int j = 0; j < 4; ++j)
    {
      const long long kn = static_cast<long long>(nx[j])*LY + ny[j];
      const int cn = plus ? static_cast<int>(kn) : -static_cast<int>(kn) - 1;
      const auto it = std::lower_bound(list.begin(), list.end(), cn);
      if(it != list.end() && *it == cn)
      {
        const int a = find(i), b = find(static_cast<int>(it - list.begin()));
        if(a != b) parent[a] = b;
      }
    }
  }
  long long plus = 0, minus = 0;
  for(int i = 0; i < count; ++i)
    if(find(i) == i) (list[i] >= 0 ? plus : minus) += 1;
  out->mean_u2 = sums[0]/N;
  out->enstrophy_density = .5*sums[1]/N;
  out->enstrophy_density_phi = sums[3] > 0 ? .5*sums[2]/sums[3] : 0.0;
  out->phi_area = sums[3];
  out->perimeter = sums[4];
  out->defects_plus = plus;
  out->defects_minus = minus;
  out->charged_sites = count;
  return 0;
}

int mass_lb_device_state(mass_lb_handle* h, void** planes, long long* plane_stride,
                         int* nplanes_out)
{
  if(!h || !planes) return fail(MASS_LB_EINVAL, "null argument");
  if(!h->fused) return fail(MASS_LB_EUNSUPPORTED, "device state view is FP32-fused only");
  *planes = h->cur;
  if(plane_stride) *plane_stride = static_cast<long long>(h->LX)*h->LY;
  if(nplanes_out) *nplanes_out = nplanes(h);
  return 0;
}

// ---- checkpoints -------------------------------------------------------------

} // extern "C"

namespace {

// Checkpoint file: a fixed header, then ff (LX*LY*9 doubles, site-major
// [k][v]), QQxx, QQyx and, for lyotropic and go-or-grow, phi and, for
// go-or-grow, m (LX*LY doubles each), all in the reference's site order
// k = y + LY*x, little-endian IEEE doubles.
struct CkptHeader
{
  char magic[8];             // "MASSLBCK"
  int32_t version;           // 2 (1: FP32 populations stored with t_v*rho added)
  int32_t model, precision;  // of the handle that wrote it
  uint32_t LX, LY, bc, npc;
  uint64_t steps;
  double ftot, ptot;
  double params[14];         // GammaQ .. conc of mass_lb_params
  uint64_t payload_doubles;
  uint64_t checksum;         // FNV-1a 64 over the payload bytes
};

uint64_t fnv1a(const void* data, size_t n, uint64_t h)
{
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for(size_t i = 0; i < n; ++i) { h ^= p[i]; h *= 1099511628211ull; }
  return h;
}

constexpr uint64_t kFnvOffset = 14695981039346656037ull;

// scalar planes after ff: Q (2), phi, m
int ckpt_scalars(int model) { return model == NEM ? 2 : model == LYO ? 3 : 4; }

void params_out(const Params& P, double* v)
{
  const double a[14] = {P.GammaQ, P.GammaP, P.xi, P.tauNem, P.tauIso, P.rho, P.friction,
                        P.AA, P.CC, P.LL, P.KK, P.zeta, P.zetaI, P.conc};
  for(int i = 0; i < 14; ++i) v[i] = a[i];
}

} // namespace

extern "C" {

int mass_lb_save(mass_lb_handle* h, const char* path)
{
  if(!h || !path) return fail(MASS_LB_EINVAL, "null argument");
  const size_t N = static_cast<size_t>(h->LX)*h->LY;
  const int nf = ckpt_scalars(h->model);
  std::vector<double> buf(N*9 + nf*N);
  {
    // FP32 populations go out as the deviations from t_v*rho the state
    // holds: exact in double, where f = deviation + t_v*rho would round
    // the deviations of sites near rest
    DeviceGuard g(h->device);
    if(int r = settle_derived(h)) return r;
    if(int r = get_primary(h, MASS_LB_FF, buf.data(), true, h->precision == MASS_LB_FP32))
      return r;
  }
  const int fields[4] = {MASS_LB_QQXX, MASS_LB_QQYX, MASS_LB_PHI, MASS_LB_M};
  for(int i = 0; i < nf; ++i)
    if(int r = mass_lb_download(h, fields[i], buf.data() + N*9 + i*N)) return r;
  CkptHeader hd{};
  std::memcpy(hd.magic, "MASSLBCK", 8);
  hd.version = 2;
  hd.model = h->model;
  hd.precision = h->precision;
  hd.LX = h->LX; hd.LY = h->LY; hd.bc = h->bc; hd.npc = h->P.npc;
  hd.steps = h->steps;
  {
    DeviceGuard g(h->device);
    if(int r = resolve_totals(h)) return r;
  }
  hd.ftot = h->ftot; hd.ptot = h->ptot;
  params_out(h->P, hd.params);
  hd.payload_doubles = buf.size();
  hd.checksum = fnv1a(buf.data(), buf.size()*sizeof(double), kFnvOffset);
  FILE* f = std::fopen(path, "wb");
  if(!f) return fail(MASS_LB_EINVAL, std::string("cannot open ") + path + " for writing");
  const bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 &&
                  std::fwrite(buf.data(), sizeof(double), buf.size(), f) == buf.size();
  const bool closed = std::fclose(f) == 0;
  if(!ok || !closed) return fail(MASS_LB_EINVAL, std::string("write failed: ") + path);
  return 0;
}

int mass_lb_load(mass_lb_handle* h, const char* path)
{
  if(!h || !path) return fail(MASS_LB_EINVAL, "null argument");
  {
    DeviceGuard g(h->device);
    if(int r = settle_derived(h)) return r;
  }
  FILE* f = std::fopen(path, "rb");
  if(!f) return fail(MASS_LB_EINVAL, std::string("cannot open ") + path);
  CkptHeader hd{};
  auto bad = [&](const std::string& why) {
    std::fclose(f);
    return fail(MASS_LB_EINVAL, std::string(path) + ": " + why);
  };
  if(std::fread(&hd, sizeof(hd), 1, f) != 1) return bad("short header");
  if(std::memcmp(hd.magic, "MASSLBCK", 8) != 0) return bad("not a mass_lb checkpoint");
  if(hd.version != 1 && hd.version != 2) return bad("unknown checkpoint version");
  if(hd.model != h->model) return bad("checkpoint of another model");
  if(hd.LX != h->LX || hd.LY != h->LY) return bad("checkpoint of another lattice size");
  const size_t N = static_cast<size_t>(h->LX)*h->LY;
  const int nf = ckpt_scalars(h->model);
  if(hd.payload_doubles != N*9 + nf*N) return bad("payload size does not match the lattice");
  std::vector<double> buf(hd.payload_doubles);
  if(std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) return bad("short payload");
  std::fclose(f);
  if(fnv1a(buf.data(), buf.size()*sizeof(double), kFnvOffset) != hd.checksum)
    return fail(MASS_LB_EINVAL, std::string(path) + ": checksum mismatch (corrupted file)");
  double* ff = buf.data();
  const double* q = buf.data() + N*9;
  // version 2 from an FP32 handle: populations as deviations from t_v*rho
  // (rho of the writer); an FP32 handle of the same rho takes them as they
  // are, anything else gets the populations
  const double rho_file = hd.params[5];
  bool raw = hd.version >= 2 && hd.precision == MASS_LB_FP32;
  if(raw && !(h->precision == MASS_LB_FP32 && h->P.rho == rho_file))
  {
    for(size_t k = 0; k < N; ++k)
      for(int v = 0; v < 9; ++v) ff[9*k + v] += Tv(v)*rho_file;
    raw = false;
  }
  if(h->model == GOG)
    if(int r = mass_lb_upload_field(h, MASS_LB_M, q + 3*N)) return r;
  if(int r = upload_state(h, ff, q, q + N, h->model != NEM ? q + 2*N : nullptr, raw)) return r;
  // continue the run the checkpoint came from: step count and the totals
  // the runtime checks compare against
  h->steps = hd.steps;
  h->tot_pending = false;   // settled before the state was replaced
  h->ftot = hd.ftot;
  h->ptot = hd.ptot;
  return 0;
}

// ---- division-model hooks --------------------------------------------------

} // extern "C"

namespace {

// host doubles in site order (k = y + LY*x) -> a device plane with ghost
// ring g and row stride EY
template<typename T>
int put_plane(mass_lb_handle* h, const double* src, T* dst, int g, int EY)
{
  const int LY = static_cast<int>(h->LY);
  const long long rows_per = std::max<long long>(1, kStageSites/LY);
  for(long long x0 = 0; x0 < h->LX; x0 += rows_per)
  {
    const int nrows = static_cast<int>(std::min<long long>(rows_per, h->LX - x0));
    const long long n = static_cast<long long>(nrows)*LY;
    CU(cudaMemcpyAsync(h->stage, src + x0*LY, n*sizeof(double), cudaMemcpyHostToDevice,
                       h->stream), "upload copy");
    k_put_scalar<T><<<blocks_for(n), 256, 0, h->stream>>>(h->stage, dst, x0, nrows, LY, g, EY);
    CU(cudaGetLastError(), "upload kernel");
  }
  return 0;
}

} // namespace

extern "C" {

int mass_lb_set_phi_source(mass_lb_handle* h, const double* rate)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  DeviceGuard g(h->device);
  CU(cudaStreamSynchronize(h->stream), "sync");
  if(!rate)
  {
    h->src_on = false;
    h->s64.src = nullptr;
    h->s32.src = nullptr;
    // go-or-grow's fused step reads its rate plane in any case
    if(h->fused && h->model == GOG)
    {
      CU(cudaMemsetAsync(h->src_fused, 0, static_cast<size_t>(h->LX)*h->LY*sizeof(float),
                         h->stream), "memset");
      CU(cudaStreamSynchronize(h->stream), "sync");
    }
    return 0;
  }
  if(h->fused)
  {
    if(!h->src_fused)
      if(int r = dalloc(h, &h->src_fused, static_cast<size_t>(h->LX)*h->LY)) return r;
    if(int r = put_plane<float>(h, rate, h->src_fused, 0, static_cast<int>(h->LY))) return r;
    if(h->cfg.nt != 32) h->tuned = false;   // re-tune among warp-strip tiles
  }
  else if(h->precision == MASS_LB_FP64)
  {
    if(!h->src64)
    {
      if(int r = dalloc(h, &h->src64, h->d.NE)) return r;
      CU(cudaMemsetAsync(h->src64, 0, h->d.NE*sizeof(double), h->stream), "memset");
    }
    if(int r = put_plane<double>(h, rate, h->src64, h->d.g, h->d.EY)) return r;
    h->s64.src = h->src64;
  }
  else
  {
    if(!h->src32)
    {
      if(int r = dalloc(h, &h->src32, h->d.NE)) return r;
      CU(cudaMemsetAsync(h->src32, 0, h->d.NE*sizeof(float), h->stream), "memset");
    }
    if(int r = put_plane<float>(h, rate, h->src32, h->d.g, h->d.EY)) return r;
    h->s32.src = h->src32;
  }
  h->src_on = true;
  CU(cudaStreamSynchronize(h->stream), "upload sync");
  return 0;
}

int mass_lb_set_phi_conservation(mass_lb_handle* h, int on, double totalphi)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  DeviceGuard g(h->device);
  // conserve_phi needs a lattice-wide phi sum between the two halves of a
  // sub-step, which the one-launch fused step does not have: the lattice
  // continues on the unfused FP32 sweeps
  if(on && h->fused)
  {
    if(h->in_ensemble)
      return fail(MASS_LB_EUNSUPPORTED, "conserve_phi is not available to ensemble runs");
    if(int r = fused_to_sweeps(h)) return r;
  }
  if(on && !h->phisum)
    if(int r = dalloc(h, &h->phisum, 1 + PHI_PARTS)) return r;
  for(int i = 0; i < 2; ++i)
  {
    if(i == 0)
    {
      h->s64.conserve_phi = on ? 1 : 0;
      h->s64.totalphi = totalphi;
      h->s64.phisum = h->phisum;
    }
    else
    {
      h->s32.conserve_phi = on ? 1 : 0;
      h->s32.totalphi = totalphi;
      h->s32.phisum = h->phisum;
    }
  }
  return 0;
}

// ---- device-side masks -------------------------------------------------------

} // extern "C"

namespace {

int ensure_masks(mass_lb_handle* h)
{
  MaskScratch& m = h->mk;
  if(m.center) return 0;
  const long long N = static_cast<long long>(h->LX)*h->LY;
  const int nb = mask_blocks(N);
  if(int r = dalloc(h, &m.block_cnt, nb)) return r;
  if(int r = dalloc(h, &m.block_off, nb)) return r;
  if(int r = dalloc(h, &m.total, 1)) return r;
  if(int r = dalloc(h, &m.center, N)) return r;
  for(int i = 0; i < 2; ++i)
  {
    if(int r = dalloc(h, &m.mask[i], N)) return r;
    CU(cudaMemsetAsync(m.mask[i], 0, N, h->stream), "memset");
  }
  return 0;
}

// phi as the step kernels of this handle hold it
template<typename F>
cudaError_t with_phi(mass_lb_handle* h, F&& f)
{
  if(h->fused)
  {
    const long long plane = static_cast<long long>(h->LX)*h->LY;
    return f(MaskView<float>{h->cur + 11*plane, static_cast<int>(h->LX), static_cast<int>(h->LY),
                             0, static_cast<int>(h->LY)});
  }
  if(h->precision == MASS_LB_FP64)
    return f(MaskView<double>{h->s64.phi, h->d.LX, h->d.LY, h->d.g, h->d.EY});
  return f(MaskView<float>{h->s32.phi, h->d.LX, h->d.LY, h->d.g, h->d.EY});
}

// the source plane of this handle's step kernels, allocated on first use
int source_plane(mass_lb_handle* h, void** plane, int* is_double, int* g, int* EY)
{
  if(h->fused)
  {
    if(!h->src_fused)
      if(int r = dalloc(h, &h->src_fused, static_cast<size_t>(h->LX)*h->LY)) return r;
    *plane = h->src_fused; *is_double = 0; *g = 0; *EY = static_cast<int>(h->LY);
  }
  else if(h->precision == MASS_LB_FP64)
  {
    if(!h->src64)
    {
      if(int r = dalloc(h, &h->src64, h->d.NE)) return r;
      CU(cudaMemsetAsync(h->src64, 0, h->d.NE*sizeof(double), h->stream), "memset");
    }
    *plane = h->src64; *is_double = 1; *g = h->d.g; *EY = h->d.EY;
  }
  else
  {
    if(!h->src32)
    {
      if(int r = dalloc(h, &h->src32, h->d.NE)) return r;
      CU(cudaMemsetAsync(h->src32, 0, h->d.NE*sizeof(float), h->stream), "memset");
    }
    *plane = h->src32; *is_double = 0; *g = h->d.g; *EY = h->d.EY;
  }
  return 0;
}

} // namespace

extern "C" {

int mass_lb_mask_candidates(mass_lb_handle* h, long long* count)
{
  if(!h || !count) return fail(MASS_LB_EINVAL, "null argument");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  DeviceGuard g(h->device);
  if(int r = ensure_masks(h)) return r;
  const cudaError_t e = with_phi(h, [&](const auto& v) { return mask_count(v, h->mk, h->stream); });
  if(e != cudaSuccess) return cuda_fail(e, "mask candidates");
  long long n = 0;
  CU(cudaMemcpyAsync(&n, h->mk.total, sizeof(n), cudaMemcpyDeviceToHost, h->stream), "count copy");
  CU(cudaStreamSynchronize(h->stream), "count sync");
  h->mk_count = n;
  *count = n;
  return 0;
}

int mass_lb_draw_mask(mass_lb_handle* h, int kind, const double* draws, long long ndraws,
                      double coef, double phi_critical, double radius, double alpha, double beta)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  if(kind != 0 && kind != 1) return fail(MASS_LB_EINVAL, "kind must be 0 (division) or 1 (death)");
  if(h->mk_count < 0) return fail(MASS_LB_EINVAL, "call mass_lb_mask_candidates first");
  if(ndraws != h->mk_count)
    return fail(MASS_LB_EINVAL, "one draw per candidate site is needed (ndraws != candidates)");
  if(ndraws > 0 && !draws) return fail(MASS_LB_EINVAL, "null draws");
  DeviceGuard g(h->device);
  MaskScratch& m = h->mk;
  // the candidate count drifts from draw to draw: buffers grow
  // geometrically, up to one draw per site
  const long long N = static_cast<long long>(h->LX)*h->LY;
  const long long cap = std::min(N, std::max(2*ndraws, 1ll << 16));
  if(ndraws > m.draws_cap)
  {
    double* p = nullptr;
    if(int r = dalloc(h, &p, static_cast<size_t>(cap))) return r;
    m.draws = p;
    m.draws_cap = cap;
  }
  if(ndraws > 0)
  {
    // through a pinned staging buffer, so that neither this copy nor the
    // caller waits for the stream; the buffer is refilled only after the
    // previous copy out of it has run
    if(!h->mk_copied)
      CU(cudaEventCreateWithFlags(&h->mk_copied, cudaEventDisableTiming), "event");
    else
      CU(cudaEventSynchronize(h->mk_copied), "staging wait");
    if(ndraws > h->mk_pinned_cap)
    {
      if(h->mk_pinned) cudaFreeHost(h->mk_pinned);
      h->mk_pinned = nullptr;
      h->mk_pinned_cap = 0;
      CU(cudaMallocHost(reinterpret_cast<void**>(&h->mk_pinned), cap*sizeof(double)),
         "pinned staging");
      h->mk_pinned_cap = cap;
    }
    std::memcpy(h->mk_pinned, draws, ndraws*sizeof(double));
    CU(cudaMemcpyAsync(m.draws, h->mk_pinned, ndraws*sizeof(double), cudaMemcpyHostToDevice,
                       h->stream), "draws copy");
    CU(cudaEventRecord(h->mk_copied, h->stream), "event");
  }
  cudaError_t e = with_phi(h, [&](const auto& v) {
    return mask_draw(v, m, kind, ndraws, coef, phi_critical, radius, h->stream);
  });
  if(e != cudaSuccess) return cuda_fail(e, "mask draw");
  void* plane = nullptr;
  int dbl = 0, gg = 0, EY = 0;
  if(int r = source_plane(h, &plane, &dbl, &gg, &EY)) return r;
  e = dbl ? mask_rate<double>(static_cast<int>(h->LX), static_cast<int>(h->LY), gg, EY, m, alpha,
                              beta, static_cast<double*>(plane), h->stream)
          : mask_rate<float>(static_cast<int>(h->LX), static_cast<int>(h->LY), gg, EY, m, alpha,
                             beta, static_cast<float*>(plane), h->stream);
  if(e != cudaSuccess) return cuda_fail(e, "mask rate");
  if(h->fused && h->cfg.nt != 32) h->tuned = false;   // the source runs in the warp-strip kernel
  h->s64.src = h->src64;
  h->s32.src = h->src32;
  h->src_on = true;
  return 0;
}

int mass_lb_get_mask(mass_lb_handle* h, int kind, unsigned char* out)
{
  if(!h || !out) return fail(MASS_LB_EINVAL, "null argument");
  if(kind != 0 && kind != 1) return fail(MASS_LB_EINVAL, "kind must be 0 (division) or 1 (death)");
  DeviceGuard g(h->device);
  const size_t N = static_cast<size_t>(h->LX)*h->LY;
  if(!h->mk.center)
  {
    std::memset(out, 0, N);
    return 0;
  }
  CU(cudaMemcpyAsync(out, h->mk.mask[kind], N, cudaMemcpyDeviceToHost, h->stream), "mask copy");
  CU(cudaStreamSynchronize(h->stream), "mask sync");
  return 0;
}

} // extern "C"

namespace {

int ensure_queue(mass_lb_handle* h)
{
  if(h->mq.buf) return 0;
  constexpr int S = mass_lb_handle::MQ_SLOTS, B = mass_lb_handle::MQ_STAGES;
  const long long N = static_cast<long long>(h->LX)*h->LY;
  const long long cap = 6*N + (1ll << 16);
  if(int r = dalloc(h, &h->mq.buf, static_cast<size_t>(cap))) return r;
  if(int r = dalloc(h, &h->mq_state, 2)) return r;
  if(int r = dalloc(h, &h->mq_snap, 2*S)) return r;
  h->mq.head = h->mq_state;
  h->mq_err = reinterpret_cast<int*>(h->mq_state + 1);   // little-endian low word
  CU(cudaMemsetAsync(h->mq_state, 0, 2*sizeof(long long), h->stream), "memset");
  CU(cudaMallocHost(reinterpret_cast<void**>(&h->mq_host), 2*S*sizeof(long long)), "pinned");
  CU(cudaStreamCreateWithFlags(&h->mq_copy, cudaStreamNonBlocking), "copy stream");
  for(int i = 0; i < 2*S; ++i) h->mq_host[i] = 0;
  for(int i = 0; i < B; ++i)
  {
    CU(cudaEventCreateWithFlags(&h->mq_copied[i], cudaEventDisableTiming), "event");
    CU(cudaEventRecord(h->mq_copied[i], h->stream), "event");
  }
  for(int i = 0; i < S; ++i)
  {
    CU(cudaEventCreateWithFlags(&h->mq_counted[i], cudaEventDisableTiming), "event");
    CU(cudaEventCreateWithFlags(&h->mq_drew[i], cudaEventDisableTiming), "event");
  }
  h->mq.cap = cap;
  h->mq.supplied = 0;
  h->mq_issued = h->mq_known = h->mq_consumed = 0;
  return 0;
}

// Read the counts of the queued draws that have landed, in order: all of
// them up to draw `until` (waiting for them), then any later ones that are
// already there.
int queue_refresh(mass_lb_handle* h, long long until)
{
  constexpr int S = mass_lb_handle::MQ_SLOTS;
  while(h->mq_known < h->mq_issued)
  {
    const int sl = static_cast<int>(h->mq_known % S);
    if(h->mq_known < until) CU(cudaEventSynchronize(h->mq_counted[sl]), "queue count");
    else
    {
      const cudaError_t e = cudaEventQuery(h->mq_counted[sl]);
      if(e == cudaErrorNotReady) break;
      CU(e, "queue count");
    }
    h->mq_consumed = h->mq_host[2*sl];
    if(h->mq_host[2*sl + 1])
      return fail(MASS_LB_EINVAL, "a queued mask needed more draws than were supplied");
    ++h->mq_known;
  }
  return 0;
}

// staging buffer i with room for n values (its previous copy has been
// read: the caller waited on mq_copied[i])
int ensure_staging(mass_lb_handle* h, int i, long long n)
{
  if(n <= h->mq_pinned_cap[i]) return 0;
  if(h->mq_pinned[i]) cudaFreeHost(h->mq_pinned[i]);
  h->mq_pinned[i] = nullptr;
  h->mq_pinned_cap[i] = 0;
  const long long cap = std::max(2*n, 1ll << 16);
  CU(cudaMallocHost(reinterpret_cast<void**>(&h->mq_pinned[i]), cap*sizeof(double)), "pinned");
  h->mq_pinned_cap[i] = cap;
  return 0;
}

} // namespace

extern "C" {

int mass_lb_mask_staging(mass_lb_handle* h, long long n, double** buf)
{
  if(!h || !buf) return fail(MASS_LB_EINVAL, "null argument");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  if(n < 0) return fail(MASS_LB_EINVAL, "bad count");
  DeviceGuard g(h->device);
  if(int r = ensure_queue(h)) return r;
  const int i = h->mq_stage;
  CU(cudaEventSynchronize(h->mq_copied[i]), "staging wait");
  if(int r = ensure_staging(h, i, n)) return r;
  *buf = h->mq_pinned[i];
  return 0;
}

int mass_lb_mask_supply(mass_lb_handle* h, const double* u, long long n)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  if(n < 0 || (n > 0 && !u)) return fail(MASS_LB_EINVAL, "bad draws");
  if(n == 0) return 0;
  DeviceGuard g(h->device);
  if(int r = ensure_queue(h)) return r;
  MaskQueue& q = h->mq;
  if(q.supplied + n - h->mq_consumed > q.cap)
  {
    if(int r = queue_refresh(h, h->mq_issued)) return r;
    if(q.supplied + n - h->mq_consumed > q.cap)
      return fail(MASS_LB_EINVAL, "mask queue full (more than 6*LX*LY + 65536 unconsumed draws)");
  }
  // a staging buffer is refilled once its previous copy has been read;
  // values written into it through mass_lb_mask_staging go up as they are
  const int i = h->mq_stage;
  const double* stage = h->mq_pinned[i];
  const bool staged = u == stage;
  if(staged && n > h->mq_pinned_cap[i])
    return fail(MASS_LB_EINVAL, "more draws than the staging buffer holds");
  CU(cudaEventSynchronize(h->mq_copied[i]), "staging wait");
  if(!staged)
  {
    if(int r = ensure_staging(h, i, n)) return r;
    stage = h->mq_pinned[i];
    std::memcpy(h->mq_pinned[i], u, n*sizeof(double));
  }
  // the values go up on the copy stream, so they need not wait for the
  // steps queued before them; the next draw on the step stream waits for them
  const long long p = q.supplied % q.cap;
  const long long n1 = std::min(n, q.cap - p);
  CU(cudaMemcpyAsync(q.buf + p, stage, n1*sizeof(double), cudaMemcpyHostToDevice,
                     h->mq_copy), "supply copy");
  if(n1 < n)
    CU(cudaMemcpyAsync(q.buf, stage + n1, (n - n1)*sizeof(double),
                       cudaMemcpyHostToDevice, h->mq_copy), "supply copy");
  CU(cudaEventRecord(h->mq_copied[i], h->mq_copy), "event");
  CU(cudaStreamWaitEvent(h->stream, h->mq_copied[i], 0), "event wait");
  h->mq_stage = i ^ 1;
  q.supplied += n;
  return 0;
}

int mass_lb_draw_masks_queued(mass_lb_handle* h, int kinds, double division_coef,
                              double division_radius, double death_coef, double death_radius,
                              double phi_critical, double alpha, double beta)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(h->model == NEM) return fail(MASS_LB_EUNSUPPORTED, "the nematic model has no phi");
  if(kinds < 1 || kinds > 3) return fail(MASS_LB_EINVAL, "kinds: bit 0 division, bit 1 death");
  DeviceGuard g(h->device);
  if(int r = ensure_masks(h)) return r;
  if(int r = ensure_queue(h)) return r;
  void* plane = nullptr;
  int dbl = 0, gg = 0, EY = 0;
  if(int r = source_plane(h, &plane, &dbl, &gg, &EY)) return r;
  // this draw's count goes to a free slot (waiting for the draw that used it)
  constexpr int S = mass_lb_handle::MQ_SLOTS;
  if(int r = queue_refresh(h, h->mq_issued - S + 1)) return r;
  const int sl = static_cast<int>(h->mq_issued % S);
  // the source plane has phi's precision
  const cudaError_t e = with_phi(h, [&](const auto& v) {
    using T = std::remove_cv_t<std::remove_pointer_t<decltype(v.phi)>>;
    if(dbl != (std::is_same<T, double>::value ? 1 : 0)) return cudaErrorInvalidValue;
    const QueuedDraw<T> w{kinds, {division_coef, death_coef}, {division_radius, death_radius},
                          phi_critical, alpha, beta, static_cast<T*>(plane), gg, EY, h->mq_err,
                          h->mq_snap + 2*sl};
    return mask_draw_queued_fused(v, h->mk, h->mq, w, h->stream);
  });
  if(e != cudaSuccess) return cuda_fail(e, "queued masks");
  // the snapshot comes down on the copy stream, off the step stream
  CU(cudaEventRecord(h->mq_drew[sl], h->stream), "event");
  CU(cudaStreamWaitEvent(h->mq_copy, h->mq_drew[sl], 0), "event wait");
  CU(cudaMemcpyAsync(h->mq_host + 2*sl, h->mq_snap + 2*sl, 2*sizeof(long long),
                     cudaMemcpyDeviceToHost, h->mq_copy), "queue count");
  CU(cudaEventRecord(h->mq_counted[sl], h->mq_copy), "event");
  ++h->mq_issued;
  if(h->fused && h->cfg.nt != 32) h->tuned = false;   // the source runs in the warp-strip kernel
  h->s64.src = h->src64;
  h->s32.src = h->src32;
  h->src_on = true;
  return 0;
}

int mass_lb_mask_consumed(mass_lb_handle* h, long long* consumed)
{
  if(!h || !consumed) return fail(MASS_LB_EINVAL, "null argument");
  DeviceGuard g(h->device);
  if(int r = queue_refresh(h, h->mq_issued)) return r;
  *consumed = h->mq_consumed;
  return 0;
}

int mass_lb_mask_progress(mass_lb_handle* h, long long* consumed, int* pending)
{
  if(!h || !consumed || !pending) return fail(MASS_LB_EINVAL, "null argument");
  DeviceGuard g(h->device);
  if(int r = queue_refresh(h, 0)) return r;
  *consumed = h->mq_consumed;
  *pending = static_cast<int>(h->mq_issued - h->mq_known);
  return 0;
}

} // extern "C"

extern "C" {

// ---- go-or-grow ------------------------------------------------------------

int mass_lb_set_go_or_grow_params(mass_lb_handle* h, const mass_lb_go_or_grow_params* p)
{
  if(!h || !p) return fail(MASS_LB_EINVAL, "null argument");
  if(h->model != GOG) return fail(MASS_LB_EUNSUPPORTED, "not a go-or-grow lattice");
  DeviceGuard g(h->device);
  if(int r = settle_derived(h)) return r;
  const Pheno ph{p->B, p->Snem, p->Dchi, p->Achi, p->Ochi, p->phiswitch, p->phi_critical,
                 p->growTogether ? 1 : 0};
  h->s64.ph = ph;
  h->s32.ph = ph;
  return 0;
}

int mass_lb_relax_free_energy(mass_lb_handle* h, unsigned steps, double dt, int relax_phi,
                              int relax_Q, double* phisum)
{
  if(!h) return fail(MASS_LB_EINVAL, "null handle");
  if(h->model != GOG) return fail(MASS_LB_EUNSUPPORTED, "not a go-or-grow lattice");
  DeviceGuard g(h->device);
  if(int r = settle_derived(h)) return r;
  // an earlier asynchronous upload's totals land first, so that they cannot
  // later overwrite the relaxed phi total assigned below
  if(int r = resolve_totals(h)) return r;
  if(!h->relaxsum)
    if(int r = dalloc(h, &h->relaxsum, 1)) return r;
  // the relaxation runs on the sweeps' state; a fused lattice goes there
  // and back
  const bool was_fused = h->fused;
  if(int r = fused_to_sweeps(h)) return r;
  const int bc = h->wall ? static_cast<int>(h->bc) : 0;
  const int r = h->precision == MASS_LB_FP64
    ? relax_unfused_f64(h->d, h->P, h->s64, bc, steps, dt, relax_phi, relax_Q, h->relaxsum, h->stream)
    : relax_unfused_f32(h->d, h->P, h->s32, bc, steps, dt, relax_phi, relax_Q, h->relaxsum, h->stream);
  if(r) return cuda_fail(cudaGetLastError(), "relaxation");
  // chi follows the relaxed phi
  const int rc = h->precision == MASS_LB_FP64 ? update_chi_f64(h->d, h->s64, h->stream)
                                              : update_chi_f32(h->d, h->s32, h->stream);
  if(rc) return cuda_fail(cudaGetLastError(), "chi update");
  double sum = 0;
  CU(cudaMemcpyAsync(&sum, h->relaxsum, sizeof(double), cudaMemcpyDeviceToHost, h->stream),
     "relaxation sum");
  CU(cudaStreamSynchronize(h->stream), "relaxation sync");
  if(was_fused)
  {
    if(int r = sweeps_to_fused(h)) return r;
    CU(cudaStreamSynchronize(h->stream), "state copy sync");
  }
  h->ptot = sum;
  h->has_prev = false;
  if(phisum) *phisum = sum;
  return 0;
}

// ---- ensembles ------------------------------------------------------------

} // extern "C"

struct mass_lb_ensemble
{
  int device = 0;
  int model = LYO;
  cudaStream_t stream = nullptr;
  std::vector<mass_lb_handle*> runs;
  std::vector<int> order;       // runs, largest first
  EnsRun* d_runs = nullptr;
  int* d_item_run = nullptr;
  int* d_counter = nullptr;
  int* d_err = nullptr;
  int nitems = 0;
  int capacity = 0;             // items the device list holds
  int rows = 0;                 // rows per chunk (0: not tuned yet)
  int slot0 = -1;
  int grid = 0;
  cudaGraphExec_t graph = nullptr;   // two steps: parity 0 then 1
  std::vector<void*> allocs;
};

namespace {

std::mutex g_slot_mu;
std::vector<unsigned char> g_slot_used[64];   // per device: constant-memory slots

int reserve_slots(int dev, int n)
{
  std::lock_guard<std::mutex> lock(g_slot_mu);
  auto& used = g_slot_used[dev & 63];
  if(used.empty()) used.assign(ENS_MAX_RUNS, 0);
  for(int s = 0; s + n <= ENS_MAX_RUNS; ++s)
  {
    bool free_run = true;
    for(int k = 0; k < n && free_run; ++k) free_run = !used[s + k];
    if(free_run)
    {
      for(int k = 0; k < n; ++k) used[s + k] = 1;
      return s;
    }
  }
  return -1;
}

void release_slots(int dev, int s, int n)
{
  std::lock_guard<std::mutex> lock(g_slot_mu);
  auto& used = g_slot_used[dev & 63];
  for(int k = 0; k < n && s >= 0; ++k) used[s + k] = 0;
}

// Pack the work items of every run (largest run first) for chunk height
// `rows`, and point each run's descriptor at its handle's current buffers
// (parity 0 reads handle->cur).
int ens_pack(mass_lb_ensemble* e, int rows)
{
  std::vector<EnsRun> desc(e->runs.size());
  std::vector<int> item_run;
  for(int r : e->order)
  {
    mass_lb_handle* h = e->runs[r];
    EnsRun& d = desc[r];
    d.a = h->cur;
    d.b = h->nxt;
    d.LX = static_cast<int>(h->LX);
    d.LY = static_cast<int>(h->LY);
    d.plane = static_cast<long long>(h->LX)*h->LY;
    d.nstrips = (d.LY + ENS_WOUT - 1)/ENS_WOUT;
    d.rows = std::min(rows, d.LX);
    d.item0 = static_cast<int>(item_run.size());
    d.slot = e->slot0 + r;
    const int n = d.nstrips*((d.LX + d.rows - 1)/d.rows);
    for(int k = 0; k < n; ++k) item_run.push_back(r);
  }
  if(static_cast<int>(item_run.size()) > e->capacity)   // sized for rows = 32
    return fail(MASS_LB_EINVAL, "ensemble item list overflow");
  e->nitems = static_cast<int>(item_run.size());
  CU(cudaMemcpyAsync(e->d_runs, desc.data(), desc.size()*sizeof(EnsRun),
                     cudaMemcpyHostToDevice, e->stream), "ensemble descriptors");
  CU(cudaMemcpyAsync(e->d_item_run, item_run.data(), item_run.size()*sizeof(int),
                     cudaMemcpyHostToDevice, e->stream), "ensemble items");
  return 0;
}

int ens_launch(mass_lb_ensemble* e, int parity)
{
  CU(cudaMemsetAsync(e->d_counter, 0, sizeof(int), e->stream), "ensemble counter");
  CU(launch_fused_warp_ensemble(e->d_runs, e->d_item_run, e->nitems, e->d_counter, e->d_err,
                                parity, e->model, e->grid, e->stream), "ensemble step");
  return 0;
}

// Choose the chunk height by timing one launch per candidate; the state is
// read from buffer a and written to b, so it does not advance.
int ens_autotune(mass_lb_ensemble* e)
{
  cudaEvent_t t0, t1;
  CU(cudaEventCreate(&t0), "event");
  CU(cudaEventCreate(&t1), "event");
  float best = 1e30f;
  int best_rows = 64;
  const int cand[] = {32, 64, 128, 256};
  for(int rows : cand)
  {
    if(int r = ens_pack(e, rows)) return r;
    if(int r = ens_launch(e, 0)) return r;
    CU(cudaEventRecord(t0, e->stream), "event");
    for(int k = 0; k < 3; ++k)
      if(int r = ens_launch(e, 0)) return r;
    CU(cudaEventRecord(t1, e->stream), "event");
    CU(cudaEventSynchronize(t1), "event");
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, t0, t1), "event");
    if(std::getenv("MASS_LB_TUNE_LOG"))
      std::fprintf(stderr, "mass_lb ensemble autotune: rows %d: %.4f ms/step\n", rows, ms/3);
    if(ms < best) { best = ms; best_rows = rows; }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  e->rows = best_rows;
  for(mass_lb_handle* h : e->runs) h->has_prev = false;   // b buffers were scratch
  return ens_pack(e, e->rows);
}

} // namespace

extern "C" {

int mass_lb_ensemble_create(int nruns, const mass_lb_params* params, const unsigned* LX,
                            const unsigned* LY, mass_lb_ensemble** out)
{
  if(!params || !LX || !LY || !out) return fail(MASS_LB_EINVAL, "null argument");
  *out = nullptr;
  if(nruns < 1) return fail(MASS_LB_EINVAL, "an ensemble needs at least one run");
  if(nruns > ENS_MAX_RUNS) return fail(MASS_LB_EINVAL, "too many runs for one ensemble");
  const int model = params[0].model;
  if(model != MASS_LB_LYOTROPIC && model != MASS_LB_NEMATIC)
    return fail(MASS_LB_EUNSUPPORTED, "ensembles run the lyotropic or nematic model");
  for(int i = 0; i < nruns; ++i)
  {
    if(params[i].model != model) return fail(MASS_LB_EINVAL, "all runs must use one model");
    if(params[i].npc != 1) return fail(MASS_LB_EUNSUPPORTED, "ensembles need npc = 1");
    if(!fused_supported(static_cast<int>(LX[i]), static_cast<int>(LY[i]), 32))
      return fail(MASS_LB_EUNSUPPORTED, "run lattice not supported by the fused kernel "
                                        "(LY % 4 == 0 and LY >= 64 required)");
  }
  auto* e = new mass_lb_ensemble();
  CU(cudaGetDevice(&e->device), "cudaGetDevice");
  e->model = model;
  auto bail = [&](int r) { mass_lb_ensemble_destroy(e); return r; };
  e->slot0 = reserve_slots(e->device, nruns);
  if(e->slot0 < 0) return bail(fail(MASS_LB_EUNSUPPORTED, "no free parameter slots on this device"));
  if(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MASS_LB_ECUDA, "stream create"));
  long long items_max = 0;
  for(int i = 0; i < nruns; ++i)
  {
    mass_lb_handle* h = nullptr;
    if(int r = mass_lb_create(&params[i], LX[i], LY[i], 0, MASS_LB_FP32, &h)) return bail(r);
    h->tuned = true;   // the ensemble kernel steps this lattice
    h->in_ensemble = true;
    e->runs.push_back(h);
    const long long strips = (LY[i] + ENS_WOUT - 1)/ENS_WOUT;
    items_max += strips*((LX[i] + 31)/32);
    if(ensemble_set_params(e->slot0 + i, p32_of(h->P), model, e->stream) != cudaSuccess)
      return bail(fail(MASS_LB_ECUDA, "ensemble parameters"));
  }
  e->order.resize(nruns);
  for(int i = 0; i < nruns; ++i) e->order[i] = i;
  std::stable_sort(e->order.begin(), e->order.end(), [&](int a, int b) {
    return static_cast<long long>(LX[a])*LY[a] > static_cast<long long>(LX[b])*LY[b];
  });
  auto dal = [&](void** p, size_t bytes) {
    if(cudaMalloc(p, bytes) != cudaSuccess) { cudaGetLastError(); return false; }
    e->allocs.push_back(*p);
    return true;
  };
  if(!dal(reinterpret_cast<void**>(&e->d_runs), nruns*sizeof(EnsRun)) ||
     !dal(reinterpret_cast<void**>(&e->d_item_run), items_max*sizeof(int)) ||
     !dal(reinterpret_cast<void**>(&e->d_counter), sizeof(int)) ||
     !dal(reinterpret_cast<void**>(&e->d_err), sizeof(int)))
    return bail(fail(MASS_LB_ENOMEM, "ensemble allocation"));
  e->capacity = static_cast<int>(items_max);
  e->grid = ensemble_grid(model);
  if(e->grid <= 0) return bail(fail(MASS_LB_ECUDA, "ensemble kernel occupancy"));
  if(cudaMemsetAsync(e->d_err, 0, sizeof(int), e->stream) != cudaSuccess)
    return bail(fail(MASS_LB_ECUDA, "memset"));
  if(const char* env = std::getenv("MASS_LB_ENSEMBLE_ROWS"))
    e->rows = std::max(1, std::atoi(env));
  *out = e;
  return 0;
}

void mass_lb_ensemble_destroy(mass_lb_ensemble* e)
{
  if(!e) return;
  DeviceGuard g(e->device);
  if(e->stream) cudaStreamSynchronize(e->stream);
  if(e->graph) cudaGraphExecDestroy(e->graph);
  for(mass_lb_handle* h : e->runs) mass_lb_destroy(h);
  for(void* p : e->allocs) cudaFree(p);
  if(e->slot0 >= 0) release_slots(e->device, e->slot0, static_cast<int>(e->runs.size()));
  if(e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

mass_lb_handle* mass_lb_ensemble_run(mass_lb_ensemble* e, int i)
{
  if(!e || i < 0 || i >= static_cast<int>(e->runs.size())) return nullptr;
  return e->runs[i];
}

int mass_lb_ensemble_size(mass_lb_ensemble* e)
{
  return e ? static_cast<int>(e->runs.size()) : 0;
}

int mass_lb_ensemble_step(mass_lb_ensemble* e, unsigned nsteps)
{
  if(!e) return fail(MASS_LB_EINVAL, "null ensemble");
  if(nsteps == 0) return 0;
  DeviceGuard g(e->device);
  // the run handles may have been uploaded or stepped on their own streams
  for(mass_lb_handle* h : e->runs)
  {
    if(h->src_on)
      return fail(MASS_LB_EUNSUPPORTED, "ensemble runs cannot carry a phi source");
    CU(cudaStreamSynchronize(h->stream), "run sync");
  }
  if(e->rows == 0)
  {
    if(int r = ens_autotune(e)) return r;
  }
  else if(int r = ens_pack(e, e->rows)) return r;
  if(!e->graph)
  {
    // one replay = two steps: a -> b, then b -> a
    cudaGraph_t gr = nullptr;
    CU(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "capture");
    int r1 = ens_launch(e, 0);
    int r2 = r1 ? r1 : ens_launch(e, 1);
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &gr);
    if(r1 || r2) { if(gr) cudaGraphDestroy(gr); return r1 ? r1 : r2; }
    CU(ce, "end capture");
    const cudaError_t ie = cudaGraphInstantiate(&e->graph, gr, 0);
    cudaGraphDestroy(gr);
    CU(ie, "graph instantiate");
  }
  for(unsigned k = 0; k + 1 < nsteps; k += 2)
    CU(cudaGraphLaunch(e->graph, e->stream), "graph launch");
  if(nsteps & 1)
    if(int r = ens_launch(e, 0)) return r;
  // an odd count leaves every run's state in b; either way the other buffer
  // holds the state one step back
  for(mass_lb_handle* h : e->runs)
  {
    if(nsteps & 1) std::swap(h->cur, h->nxt);
    h->has_prev = true;
    h->steps += nsteps;
  }
  CU(cudaStreamSynchronize(e->stream), "ensemble sync");
  int err = 0;
  CU(cudaMemcpy(&err, e->d_err, sizeof(int), cudaMemcpyDeviceToHost), "ensemble err");
  if(err) return fail(MASS_LB_ECUDA, "ensemble step: a bounded wait on a bulk copy timed out");
  return 0;
}

int mass_lb_ensemble_get_rows(mass_lb_ensemble* e)
{
  return e ? e->rows : 0;
}

} // extern "C"
