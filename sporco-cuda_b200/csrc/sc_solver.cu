// Host driver of the CBPDN solvers: planning, workspace layout, launch
// sequence, and the C ABI (native sc_* layer + reference-compatible layer).
//
// The reference's drivers (sporco_cuda/src/cbpdn.cu:86-616 and
// cbpdn_grd.cu:97-658) allocate 9 full-size arrays, build cuFFT plans and
// drive every ADMM iteration from the host with two device synchronisations
// and managed-memory reads per iteration.  Here the iteration runs entirely
// on the device: rho, the residuals and the stopping decision live in device
// memory (ImgState), and the host only polls a "finished" counter every
// `check_every` iterations.  State per image is Y, U (real) and one spectrum
// array; the dictionary spectrum is shared by the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sporco_b200.h"
#include "sc_aux_kernels.cuh"
#include "sc_dispatch.cuh"

#define SC_VERSION "0.1.0"

// ------------------------------------------------------------- error state --
static thread_local int g_last_status = SC_OK;
static thread_local char g_last_error[512] = "";

static int set_status(int st, const char* fmt, ...) {
  g_last_status = st;
  if (fmt) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
  } else {
    g_last_error[0] = 0;
  }
  return st;
}

#define CU_TRY(call)                                                          \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return set_status(e_ == cudaErrorMemoryAllocation ? SC_ERR_OOM : SC_ERR_CUDA, \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                  \
  } while (0)

int sc_set_status_external(int st, const char* msg) { return set_status(st, msg && *msg ? "%s" : nullptr, msg); }

static std::atomic<unsigned long long> g_launches{0};
// Bumped by sc_cancel; a solve that sees it change stops launching.
static std::atomic<unsigned> g_cancel_gen{0};
extern "C" void sc_cancel(void) { g_cancel_gen.fetch_add(1); }
static thread_local sc_profile g_profile = {};

extern "C" unsigned long long sc_launch_count(void) { return g_launches.load(); }
extern "C" int sc_last_profile(sc_profile* out) {
  if (!out) return SC_ERR_INVALID;
  *out = g_profile;
  return SC_OK;
}

extern "C" int sc_last_status(void) { return g_last_status; }
extern "C" const char* sc_last_error(void) { return g_last_error; }
extern "C" const char* sc_version(void) { return SC_VERSION; }

// ------------------------------------------------------------------ planning --
static int make_fft_plan(int n, FftPlan* p) {
  memset(p, 0, sizeof(*p));
  p->n = n;
  int m = n, a = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  int q = a / 3, r = a % 3;
  for (int i = 0; i < q; ++i) p->radix[p->npass++] = 8;
  if (r == 1) p->radix[p->npass++] = 2;
  if (r == 2) p->radix[p->npass++] = 4;
  while (m % 3 == 0) { m /= 3; p->radix[p->npass++] = 3; }
  while (m % 5 == 0) { m /= 5; p->radix[p->npass++] = 5; }
  for (int f = 7; m > 1; f += 2) {
    while (m % f == 0) {
      m /= f;
      if (p->npass >= SC_FFT_MAX_PASS) return -1;
      p->radix[p->npass++] = f;
    }
    if (f * f > m && m > 1) {
      if (p->npass >= SC_FFT_MAX_PASS) return -1;
      p->radix[p->npass++] = m;
      m = 1;
    }
  }
  return 0;
}

static int pow2ceil(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Threads per transform of length n on the runtime-plan path: a power of
// two >= 32 with n <= MAXE*g.
static int group_size(int n) {
  int g = pow2ceil((n + SC_MAXE - 1) / SC_MAXE);
  return std::max(32, g);
}

#define SC_CASE_LABEL(n) case n:

static bool spec_row(int n) {
  switch (n) { SC_SPEC_ROW(SC_CASE_LABEL) return true; default: return false; }
}
static bool spec_col(int n) {
  switch (n) { SC_SPEC_COL(SC_CASE_LABEL) return true; default: return false; }
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// CTAs per image of the functional's reduction kernels (statistics only).
#define SC_OBJ_BLOCKS 128

struct Plan {
  Geom g;
  FftPlan pw, ph;
  // hot row kernels (iteration, fix-up): compile-time plan when available
  int row_g, row_nblk;
  size_t row_smem, row_smem_two, row_smem_tool;  // per CTA: V / fix-up, Y and U, tools
  // setup row kernels: runtime plan
  int rowg_g;
  size_t rowg_smem;
  // hot column kernel (solve) and setup column kernels
  int col_g, col_ntiles, col_NT, Hs;
  size_t col_smem;
  int col_hlen;
  int colg_g, colg_NT;
  size_t colg_smem, colt_smem;
  int max_iter;
  size_t off_U, off_F, off_Dh, off_Sh, off_Ps, off_E, off_twW, off_twH, off_part, off_st,
      off_it, off_xi, off_ndone, off_objspec, off_objpart, total;
};

// Process-wide caches of this file (kernel attributes, occupancy answers,
// autotuned cluster sizes, FFT-tool twiddles, SM counts) are shared by every
// host thread and guarded by this mutex; the solves themselves keep all of
// their state in the caller's workspace.
static std::mutex g_cache_mu;

#define SC_MAX_DEVICES 64
static std::atomic<int> g_num_sms[SC_MAX_DEVICES];

// SM count of the current device (cached per device).
static int num_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev >= SC_MAX_DEVICES) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }
  int n = g_num_sms[dev].load();
  if (n == 0) {
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
    g_num_sms[dev].store(n);
  }
  return n;
}

static int plan_geometry(int B, int M, int H, int W, Plan* pl) {
  if (B < 1 || M < 1 || H < 1 || W < 1)
    return set_status(SC_ERR_INVALID, "sizes must be positive (B=%d M=%d H=%d W=%d)", B, M, H, W);
  if (W > SC_MAX_N || H > 2048)
    return set_status(SC_ERR_UNSUPPORTED, "image %dx%d exceeds this build's limits (H<=2048, W<=%d)",
                      H, W, SC_MAX_N);
  Geom& g = pl->g;
  g.B = B; g.M = M; g.H = H; g.W = W;
  g.Wf = W / 2 + 1;
  g.Wp = (g.Wf + 3) & ~3;
  if (make_fft_plan(W, &pl->pw) || make_fft_plan(H, &pl->ph))
    return set_status(SC_ERR_UNSUPPORTED, "cannot factor %d or %d", W, H);
  const bool srow = spec_row(W), scol = spec_col(H);
  const int zlen = srow ? ct_len(W, row_radix(W), 1) : W;
  pl->row_g = srow ? ct_threads(W, row_radix(W)) : group_size(W);
  const int S = SC_ROW_THREADS / pl->row_g;
  const long rows = (long)M * H;
  const long npairs = (rows + 1) / 2;
  long want = (npairs + S - 1) / S;
  long cap = std::max(1L, (long)num_sms() * 8 / B);
  pl->row_nblk = (int)std::min(want, cap);
  pl->row_smem = (size_t)S * row_slot_bytes(ROW_ITER, zlen, W, g.Wp);
  pl->row_smem_two = (size_t)S * row_slot_bytes(ROW_ITER_YU, zlen, W, g.Wp);
  pl->row_smem_tool = (size_t)S * row_slot_bytes(ROW_FWD_REAL, zlen, W, g.Wp);
  pl->rowg_g = group_size(W);
  pl->rowg_smem = (size_t)(SC_ROW_THREADS / pl->rowg_g) * row_slot_bytes(ROW_FWD_REAL, W, W, g.Wp);

  pl->Hs = H + 1;
  pl->col_ntiles = (g.Wf + SC_COL_TILE - 1) / SC_COL_TILE;
  pl->col_g = scol ? ct_threads(H, col_radix(H)) : group_size(H);
  pl->col_NT = SC_COL_TILE * pl->col_g;
  pl->col_hlen = scol ? ct_len(H, col_radix(H), SC_COL_TILE) : H;
  pl->col_smem = col_smem_bytes(COL_SOLVE, pl->col_hlen);
  pl->colg_g = group_size(H);
  pl->colg_NT = SC_COL_TILE * pl->colg_g;
  pl->colg_smem = col_smem_bytes(COL_FWD, H);
  pl->colt_smem = col_smem_bytes(COL_FWD, scol ? ct_len(H, col_radix(H), SC_COL_TILE) : H);
  return SC_OK;
}

static int plan_problem(const sc_problem* p, const sc_options* o, Plan* pl) {
  int st = plan_geometry(p->B, p->M, p->H, p->W, pl);
  if (st) return st;
  if (p->Kr < 1 || p->Kc < 1 || p->Kr > p->H || p->Kc > p->W)
    return set_status(SC_ERR_INVALID, "filter size %dx%d invalid for image %dx%d", p->Kr, p->Kc,
                      p->H, p->W);
  if (o->max_iter < 0) return set_status(SC_ERR_INVALID, "max_iter < 0");
  pl->max_iter = o->max_iter;
  const Geom& g = pl->g;
  const size_t real_img = (size_t)g.M * g.H * g.W;
  const size_t spec_img = (size_t)g.M * g.H * g.Wp;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t r = off; off = align256(off + bytes); return r; };
  pl->off_U = take(sizeof(float) * real_img * g.B);
  pl->off_F = take(sizeof(float2) * spec_img * g.B);
  pl->off_Dh = take(sizeof(float2) * spec_img);
  pl->off_Sh = take(sizeof(float2) * (size_t)g.H * g.Wp * g.B);
  pl->off_Ps = take(sizeof(float) * (size_t)g.H * g.Wp);
  pl->off_E = take(sizeof(float4) * (size_t)g.M * p->Kr * g.Wp);
  pl->off_twW = take(sizeof(float2) * g.W);
  pl->off_twH = take(sizeof(float2) * g.H);
  pl->off_part = take(sizeof(double) * 5 * (size_t)pl->row_nblk * g.B);
  pl->off_st = take(sizeof(ImgState) * g.B);
  pl->off_it = take(o->record_itstat ? sizeof(double) * SC_ITSTAT_FIELDS *
                                          (size_t)std::max(1, o->max_iter) * g.B
                                    : 0);
  // the functional at Y (statistics only): Y's spectra, partial sums
  pl->off_objspec = take(o->record_itstat ? sizeof(float2) * spec_img * g.B : 0);
  pl->off_objpart = take(o->record_itstat ? sizeof(double) * 3 * SC_OBJ_BLOCKS * g.B : 0);
  pl->off_xi = take(sizeof(double) * g.B);
  pl->off_ndone = take(sizeof(int));
  pl->total = off;
  return SC_OK;
}

extern "C" size_t sc_workspace_size(const sc_problem* p, const sc_options* o) {
  Plan pl;
  if (plan_problem(p, o, &pl)) return 0;
  return pl.total;
}

// --------------------------------------------------------------- launchers --
// (the kernel tables row_fn / col_fn: sc_dispatch.cuh)

// Opt every kernel instantiation into large dynamic shared memory (the
// device's opt-in maximum) once per device.
static int prepare_fn(const void* fn, bool cluster) {
  struct Done { int dev; const void* fn; };
  static std::vector<Done> done;
  int dev = 0, optin = 0;
  CU_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (const Done& d : done)
    if (d.dev == dev && d.fn == fn) return SC_OK;
  CU_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  CU_TRY(cudaFuncGetAttributes(&fa, fn));
  CU_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - (int)fa.sharedSizeBytes));
  if (cluster) CU_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  done.push_back({dev, fn});
  return SC_OK;
}

// Hot row modes (iteration, fix-up) use the compile-time plan when the row
// length has one; the setup modes always use the runtime plan.
// Programmatic dependent launch of the solver's kernels (each waits for the
// kernel before it at its start), on request: SPORCO_B200_PDL=1.  The next
// kernel's CTAs are then scheduled while the previous one drains, which hides
// the launch gaps between the short kernels of small problems (256x256,
// M=64: 15 500 -> 16 200 iterations/s) but slowed the 512x512, M=100
// gradient and masked solves (3 030 -> 2 770), so plain launches are the
// default.
static bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("SPORCO_B200_PDL");
    return e && e[0] == '1';
  }();
  return on;
}
static void set_pdl(cudaLaunchAttribute* a) {
  a->id = cudaLaunchAttributeProgrammaticStreamSerialization;
  a->val.programmaticStreamSerializationAllowed = 1;
}

template <int MODE>
static int launch_row(const Plan& pl, RowParams rp, int B, cudaStream_t s, int nblk = 0) {
  const bool hot = row_specialised(MODE) && spec_row(rp.g.W);
  RowFn fn = row_fn<MODE>(rp.g.W);
  int st = prepare_fn((const void*)fn, false);
  if (st) return st;
  rp.gsz = hot ? pl.row_g : pl.rowg_g;
  rp.nblk = nblk > 0 ? nblk : pl.row_nblk;
  dim3 grid(rp.nblk, B);
  const size_t smem = (MODE == ROW_ITER || MODE == ROW_FIXUP) ? pl.row_smem
                      : (MODE == ROW_ITER_YU || MODE == ROW_ADJ) ? pl.row_smem_two
                      : hot ? pl.row_smem_tool : pl.rowg_smem;
  // one slot (row pair in flight) per rp.gsz threads
  const int threads = (SC_ROW_THREADS / rp.gsz) * rp.gsz;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  set_pdl(&attr[0]);
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  CU_TRY(cudaLaunchKernelEx(&cfg, fn, rp));
  ++g_launches;
  return SC_OK;
}

// Clusters of G CTAs of fn (NT threads, smem bytes each) the device keeps
// resident at once; cached per (device, function, G, smem).
static int resident_clusters(const void* fn, int NT, size_t smem, int G, int* out) {
  struct Entry { int dev; const void* fn; int G; size_t smem; int n; };
  static std::vector<Entry> cache;
  int dev = 0;
  CU_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (const Entry& e : cache)
    if (e.dev == dev && e.fn == fn && e.G == G && e.smem == smem) {
      *out = e.n;
      return SC_OK;
    }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G, 1, 1);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
    cudaGetLastError();  // a cluster size this device does not offer: none resident
    n = 0;
  }
  cache.push_back({dev, fn, G, smem, n});
  *out = n;
  return SC_OK;
}

// Cluster sizes the column pass is launched with (the model's and the
// autotuner's candidates).  Clusters lie within a GPC; with one CTA per SM a
// size that divides the GPCs' SM counts badly leaves SMs idle, which sizes
// other than the powers of two can avoid.
static const int kClusterSizes[] = {8, 6, 4, 3, 2};

// CTAs per cluster of a clustered column launch over `units` column tiles
// (tiles x images).  Candidates kClusterSizes (at most M); the estimated time
// is (maps per CTA) x (rounds of resident clusters over the units), ties go
// to the larger cluster.  Larger clusters split the maps more finely, smaller
// ones pack the GPCs more tightly.
static int cluster_size(const void* fn, int NT, size_t smem, int M, long units, int* G_out) {
  int best = std::min(8, M);
  long best_cost = -1;
  for (int G : kClusterSizes) {
    if (G > M) continue;
    int nc = 0;
    int st = resident_clusters(fn, NT, smem, G, &nc);
    if (st) return st;
    if (nc < 1) continue;
    const long cost = (long)((M + G - 1) / G) * ((units + nc - 1) / nc);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = G;
    }
  }
  *G_out = std::max(1, best);
  return SC_OK;
}

// Cluster sizes measured by the autotuner, per (device, kernel, image size,
// maps); they replace the occupancy model's choice for that shape whatever
// the number of images, so that a batch and a single solve of one size use
// the same cluster size (the map reduction's summation order depends on it).
struct TunedG {
  int dev;
  const void* fn;  // the kernel of the default radix (the key)
  int H, W, M;
  int G;
  int rm;          // column-transform radix (8, or the default col_radix(H))
  int tw;          // columns per tile (SC_COL_TILE, or 2)
  int G2;          // > 0: the tiles of the last, partly filled round of
                   // clusters of G run as a second launch with clusters of G2
};
static std::vector<TunedG> g_tuned;

// The autotuner runs unless SPORCO_B200_AUTOTUNE is set to 0; set to
// "verbose" it also reports its trial times on stderr.
static bool autotune_enabled() {
  const char* e = getenv("SPORCO_B200_AUTOTUNE");
  return !(e && e[0] == '0');
}
static bool autotune_verbose() {
  const char* e = getenv("SPORCO_B200_AUTOTUNE");
  return e && strcmp(e, "verbose") == 0;
}

// SPORCO_B200_COL_CLUSTER=G fixes the column pass's cluster size (no model,
// no autotuner) where G CTAs fit (e.g. to profile a process with the cluster
// size an unprofiled run chose); 0 or unset: no override.
static int forced_cluster(int M) {
  const char* e = getenv("SPORCO_B200_COL_CLUSTER");
  if (!e || !*e) return 0;
  const int G = atoi(e);
  return G >= 1 && G <= 16 ? std::min(G, M) : 0;
}

// SPORCO_B200_COL_TILE=2 or 4 fixes the tile width of the column pass where
// that variant is compiled (elsewhere it is ignored); 0 or unset: the tuned
// choice.
static int forced_tile() {
  const char* e = getenv("SPORCO_B200_COL_TILE");
  if (!e || !*e) return 0;
  const int tw = atoi(e);
  return tw == 2 || tw == SC_COL_TILE ? tw : 0;
}

// SPORCO_B200_COL_RADIX=8 takes the radix-8 column plans where they are
// compiled (lengths 512, 768, 1024; elsewhere it is ignored); 0 or unset:
// the tuned choice.
static int forced_radix() {
  const char* e = getenv("SPORCO_B200_COL_RADIX");
  return e && atoi(e) == 8 ? 8 : 0;
}

// SPORCO_B200_COL_SPLIT=G2 splits the column pass's partly filled last
// round of clusters off into a launch with clusters of G2 (where it applies;
// 0 or unset: the tuned choice).
static int forced_split() {
  const char* e = getenv("SPORCO_B200_COL_SPLIT");
  if (!e || !*e) return -1;
  const int G2 = atoi(e);
  return G2 >= 1 && G2 <= 16 ? G2 : -1;
}

static bool tuned_size(const void* fn, const Geom& g, int* G, int* rm = nullptr,
                       int* tw = nullptr, int* G2 = nullptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (const TunedG& e : g_tuned)
    if (e.dev == dev && e.fn == fn && e.H == g.H && e.W == g.W && e.M == g.M) {
      *G = e.G;
      if (rm) *rm = e.rm;
      if (tw) *tw = e.tw;
      if (G2) *G2 = e.G2;
      return true;
    }
  return false;
}

// Threads per column, threads per CTA and shared-memory slots per column of
// the compiled column transform of length H with radix rm, tiles of tw
// columns.
struct ColShape {
  int g, NT, hlen;
};
static ColShape col_shape(int H, int rm, int tw = SC_COL_TILE) {
  const int g = ct_threads(H, rm);
  return {g, tw * g, ct_len(H, rm, tw)};
}

// force_G > 0: launch with that cluster size, force_rm > 0 with that column
// radix, force_tw > 0 with tiles of that many columns, force_G2 >= 0 with
// that tail split (0: none; see TunedG) (the autotuner's trials); otherwise
// the tuned choice for the shape, else the occupancy model's cluster size at
// the default radix and tile.
template <int MODE>
static int launch_col(const Plan& pl, ColParams cp, int B, cudaStream_t s, int force_G = 0,
                      int force_rm = 0, int force_tw = 0, int force_G2 = -1) {
  cp.Hs = pl.Hs;
  cp.tile0 = 0;
  if (col_clustered(MODE)) {
    const ColFn fn0 = col_fn<MODE>(cp.g.H);  // default radix and tile: the tuning key
    int G = force_G > 0 ? force_G : forced_cluster(cp.g.M);
    if (force_G2 < 0) force_G2 = forced_split();
    int rm = force_rm, tw = force_tw, G2 = force_G2 > 0 ? force_G2 : 0;
    if (G <= 0) {
      int tG = 0, trm = 0, ttw = 0, tG2 = 0;
      if (tuned_size((const void*)fn0, cp.g, &tG, &trm, &ttw, &tG2)) {
        G = tG;
        if (rm <= 0) rm = trm;
        if (tw <= 0) tw = ttw;
        if (force_G2 < 0) G2 = tG2;
      }
    }
    if (force_rm <= 0 && forced_radix() > 0 && col_fn_variant<MODE>(cp.g.H, 8, SC_COL_TILE))
      rm = 8;
    if (rm <= 0) rm = col_radix(cp.g.H);
    if (force_tw <= 0) {
      const int ftw = forced_tile();
      if (ftw > 0 && col_fn_variant<MODE>(cp.g.H, rm, ftw)) tw = ftw;
    }
    if (tw <= 0) tw = SC_COL_TILE;
    ColFn fn = fn0;
    ColShape sh{pl.col_g, pl.col_NT, pl.col_hlen};
    if (rm != col_radix(cp.g.H) || tw != SC_COL_TILE) {
      fn = col_fn_variant<MODE>(cp.g.H, rm, tw);
      if (!fn)
        return set_status(SC_ERR_INVALID, "no radix-%d column plan with %d-column tiles at %d",
                          rm, tw, cp.g.H);
      sh = col_shape(cp.g.H, rm, tw);
    }
    int st = prepare_fn((const void*)fn, true);
    if (st) return st;
    const size_t smem = col_smem_bytes(MODE, sh.hlen, tw, sh.NT);
    const int ntiles = (cp.g.Wf + tw - 1) / tw;
    const long units = (long)ntiles * B;
    if (G > 0 && force_G <= 0) {
      int n = 0;  // an override or a tuned size only where such a cluster fits
      if ((st = resident_clusters((const void*)fn, sh.NT, smem, G, &n))) return st;
      if (n < 1) G = 0;
    }
    if (G <= 0 && (st = cluster_size((const void*)fn, sh.NT, smem, cp.g.M, units, &G)))
      return st;
    cp.gsz = sh.g;
    // Tail split: the tiles past the last full round of one image's
    // resident clusters of G run as a second launch with clusters of G2
    // (fewer maps per CTA), where all of them are resident at once.  Every
    // image of a batch is split at the same tile, so that a batch sums the
    // maps of every tile in the same order as a single solve.
    int t1 = ntiles;
    if (G2 > G) {
      int n1 = 0, n2 = 0;
      if ((st = resident_clusters((const void*)fn, sh.NT, smem, G, &n1))) return st;
      if ((st = resident_clusters((const void*)fn, sh.NT, smem, G2, &n2))) return st;
      const int t = n1 > 0 ? ntiles / n1 * n1 : ntiles;
      if (n1 > 0 && t > 0 && t < ntiles && ntiles - t <= n2) t1 = t;
    }
    for (int part = 0; part < 2; ++part) {
      const int Gp = part ? G2 : G;
      const int ntl = part ? ntiles - t1 : t1;
      if (ntl <= 0) continue;
      cp.G = Gp;
      cp.tile0 = part ? t1 : 0;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(Gp, ntl, B);
      cfg.blockDim = dim3(sh.NT);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = s;
      cudaLaunchAttribute attr[2];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = Gp;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      set_pdl(&attr[1]);
      cfg.attrs = attr;
      cfg.numAttrs = pdl_enabled() ? 2 : 1;
      CU_TRY(cudaLaunchKernelEx(&cfg, fn, cp));
      ++g_launches;
    }
  } else {
    // forward / inverse only: maps split 8 ways, no cluster
    ColFn fn = col_fn<MODE>(cp.g.H);
    int st = prepare_fn((const void*)fn, false);
    if (st) return st;
    const bool hot = spec_col(cp.g.H);
    cp.gsz = hot ? pl.col_g : pl.colg_g;
    cp.G = std::min(8, cp.g.M);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cp.G, pl.col_ntiles, B);
    cfg.blockDim = dim3(hot ? pl.col_NT : pl.colg_NT);
    cfg.dynamicSmemBytes = hot ? pl.colt_smem : pl.colg_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    set_pdl(&attr[0]);
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    CU_TRY(cudaLaunchKernelEx(&cfg, fn, cp));
    ++g_launches;
  }
  return SC_OK;
}

static void carve(const Plan& pl, unsigned char* ws, float** U, float2** F, float2** Dh,
                  float2** Sh, float2** twW, float2** twH, double** part, ImgState** st,
                  double** it, double** xi, int** ndone) {
  *U = (float*)(ws + pl.off_U);
  *F = (float2*)(ws + pl.off_F);
  *Dh = (float2*)(ws + pl.off_Dh);
  *Sh = (float2*)(ws + pl.off_Sh);
  *twW = (float2*)(ws + pl.off_twW);
  *twH = (float2*)(ws + pl.off_twH);
  *part = (double*)(ws + pl.off_part);
  *st = (ImgState*)(ws + pl.off_st);
  *it = (double*)(ws + pl.off_it);
  *xi = (double*)(ws + pl.off_xi);
  *ndone = (int*)(ws + pl.off_ndone);
}

__global__ void xi_kernel(double* xi, const float* lam, int B, float target, int std_res) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  double v;
  if (target > 0.f) v = target;
  else if (std_res) v = 1.0;
  else {
    const double l = lam[b];
    v = l > 0.0 ? 1.0 + pow(18.3, log10(l) + 1.0) : 1.0;
  }
  xi[b] = v;
}

extern "C" void sc_options_from_algopt(const AlgOpt* a, sc_options* o) {
  memset(o, 0, sizeof(*o));
  o->max_iter = a->MaxMainIter;
  o->relax = a->RelaxParam;
  o->abs_tol = a->AbsStopTol;
  o->rel_tol = a->RelStopTol;
  o->auto_rho = a->AutoRho;
  o->auto_rho_period = a->AutoRhoPeriod > 0 ? a->AutoRhoPeriod : 1;
  o->rho_scaling = a->RhoScaling;
  o->rsdl_ratio = a->RhoRsdlRatio;
  o->rsdl_target = a->RhoRsdlTarget;
  o->auto_scaling = a->AutoRhoScaling;
  o->std_residuals = a->StdResiduals;
  o->record_itstat = a->Verbose ? 1 : 0;
  o->check_every = 32;
  o->nonneg = a->NonNegCoef > 0 ? 1 : 0;
  o->no_bndry_cross = a->NoBndryCross > 0 ? 1 : 0;
}

// One solve of a batch of equal-sized images: set-up, iteration launches in
// chunks, host polling of the "finished" counter between chunks, results.
// sc_cbpdn_solve drives one; sc_cbpdn_solve_batch interleaves several on
// their own streams.
struct Solve {
  const sc_problem* p = nullptr;
  const sc_options* o = nullptr;
  Plan pl;
  cudaStream_t s = nullptr;
  float* U = nullptr;
  float2 *F = nullptr, *Dh = nullptr, *Sh = nullptr, *twW = nullptr, *twH = nullptr;
  double *part = nullptr, *it = nullptr, *xi = nullptr;
  ImgState* sts = nullptr;
  int* ndone = nullptr;
  float* Psum = nullptr;
  void* wsbase = nullptr;
  bool per_map_d = false, can_stop = false, finished = false;
  // State V = Y + U in the U array (row_kernel<ROW_ITER>), Y written by
  // result(); with a warm start Y and U are kept apart (ROW_ITER_YU).
  bool vstate = true;
  int col_mode = COL_SOLVE_P;  // the column solve of the iteration
  int force_G = 0;             // > 0: the column pass's cluster size (the unrolled solve)
  bool tune = true;            // run the column-pass autotuner at set-up
  unsigned gen0 = 0;           // cancellation generation at set-up
  bool cancelled = false;
  cudaEvent_t pace[2] = {nullptr, nullptr};
  int nchunk = 0;
  int done_iters = 0;
  RowParams rp = {};
  ColParams cp = {};
  FinParams fp = {};

  int setup(const sc_problem* p_, const sc_options* o_, void* workspace, size_t workspace_bytes,
            cudaStream_t stream) {
    p = p_;
    o = o_;
    s = stream;
    gen0 = g_cancel_gen.load();
    if (!p || !o) return set_status(SC_ERR_INVALID, "null problem or options");
    int st = plan_problem(p, o, &pl);
    if (st) return st;
    if (!workspace || workspace_bytes < pl.total)
      return set_status(SC_ERR_WORKSPACE, "workspace of %zu bytes needed", pl.total);
    if (((uintptr_t)workspace) & 255)
      return set_status(SC_ERR_WORKSPACE, "workspace not 256-byte aligned");
    if (!p->D || !p->S || !p->lmbda || !p->rho0 || !p->Y)
      return set_status(SC_ERR_INVALID, "null device pointer");
    if (p->grd && !p->wgrd) return set_status(SC_ERR_INVALID, "grd problem without GradWeight");
    if (p->l1_kind != SC_L1_SCALAR && !p->l1w)
      return set_status(SC_ERR_INVALID, "missing L1Weight");
    if ((p->W % 4) == 0 && (((uintptr_t)p->Y) & 15))
      return set_status(SC_ERR_INVALID, "Y must be 16-byte aligned");
    const Geom& g = pl.g;
    wsbase = workspace;
    carve(pl, (unsigned char*)workspace, &U, &F, &Dh, &Sh, &twW, &twH, &part, &sts, &it, &xi,
          &ndone);
    Psum = (float*)((unsigned char*)workspace + pl.off_Ps);
    // one d for every map unless GradWeight differs between maps
    per_map_d = p->grd && !p->wgrd_uniform;
    vstate = p->U0 == nullptr;
    // Plain problems with short filters (Kr <= 16 rows) and a compiled column
    // length take the convolution column solve.
    col_mode = per_map_d ? COL_SOLVE_W
               : (p->grd && spec_col(pl.g.H) && p->Kr <= 16) ? COL_SOLVE_G16
               : p->grd  ? COL_SOLVE
               : (spec_col(pl.g.H) && p->Kr <= 8)  ? COL_SOLVE_C8
               : (spec_col(pl.g.H) && p->Kr <= 16) ? COL_SOLVE_C16
                                                   : COL_SOLVE_P;
    float4* Erows = (float4*)((unsigned char*)workspace + pl.off_E);

    // warm_start 2: the spectra of D and S in the workspace are still valid
    const bool spectra = o->warm_start != 2;
    if (spectra) {
      twiddle_kernel<<<(g.W + 255) / 256, 256, 0, s>>>(twW, g.W);
      twiddle_kernel<<<(g.H + 255) / 256, 256, 0, s>>>(twH, g.H);
      CU_TRY(cudaGetLastError());
      g_launches += 2;
    }

    // Dictionary spectrum: rfft2 of the zero-padded filters (cuda_Pad_Dict +
    // R2C, cbpdn.cu:277-289), computed without materialising the padding.
    if (spectra) {
      RowParams r = {};
      r.g = g; r.g.B = 1;
      r.pw = pl.pw; r.twW = twW; r.F = Dh; r.D = p->D; r.Kr = p->Kr; r.Kc = p->Kc;
      if ((st = launch_row<ROW_FWD_DICT>(pl, r, 1, s))) return st;
      // the row spectra of the filter rows, before the column transform
      {
        const size_t ne = (size_t)g.M * p->Kr * g.Wp;
        filter_rows_kernel<<<(unsigned)std::min<size_t>((ne + 255) / 256, 4096), 256, 0, s>>>(
            Dh, Erows, g.M, p->Kr, g.H, g.Wp);
        CU_TRY(cudaGetLastError());
        ++g_launches;
      }
      ColParams c = {};
      c.g = g; c.g.B = 1; c.ph = pl.ph; c.twH = twH; c.twW = twW; c.F = Dh;
      if ((st = launch_col<COL_FWD>(pl, c, 1, s))) return st;
      const size_t plane = (size_t)g.H * g.Wp;
      psum_kernel<<<(unsigned)((plane + 255) / 256), 256, 0, s>>>(Dh, Psum, g.M, plane);
      CU_TRY(cudaGetLastError());
      ++g_launches;
    }
    // Signal spectra (B images, one map each).
    if (spectra) {
      RowParams r = {};
      r.g = g; r.g.M = 1;
      r.pw = pl.pw; r.twW = twW; r.F = Sh; r.src = p->S;
      const long npairs = ((long)g.H + 1) / 2;
      const int S = SC_ROW_THREADS / pl.rowg_g;
      const int nb = (int)std::max(1L, std::min((npairs + S - 1) / S, (long)num_sms()));
      if ((st = launch_row<ROW_FWD_REAL>(pl, r, g.B, s, nb))) return st;
      ColParams c = {};
      c.g = g; c.g.M = 1; c.ph = pl.ph; c.twH = twH; c.twW = twW; c.F = Sh;
      if ((st = launch_col<COL_FWD>(pl, c, g.B, s))) return st;
    }
    if (o->warm_start) {
      // continue the state an earlier solve of this problem left in the
      // workspace: iterates, spectra of Y - U, rho, iteration count
      warm_state_kernel<<<(g.B + 127) / 128, 128, 0, s>>>(sts, g.B, ndone);
    } else {
      if ((st = init_iterates())) return st;
      init_state_kernel<<<(g.B + 127) / 128, 128, 0, s>>>(sts, p->rho0, g.B, ndone);
    }
    xi_kernel<<<(g.B + 127) / 128, 128, 0, s>>>(xi, p->lmbda, g.B, o->rsdl_target,
                                                 o->std_residuals);
    CU_TRY(cudaGetLastError());
    g_launches += 2;

    rp.g = g; rp.pw = pl.pw; rp.twW = twW; rp.F = F; rp.Y = p->Y; rp.Yo = p->Y; rp.U = U;
    rp.lam = p->lmbda; rp.l1_kind = p->l1_kind; rp.l1_scalar = p->l1_scalar; rp.l1w = p->l1w;
    rp.mask = p->mask; rp.relax = o->relax; rp.invN = (float)(1.0 / ((double)g.H * g.W));
    rp.nonneg = o->nonneg ? 1 : 0;
    rp.bnd_r = o->no_bndry_cross && p->Kr > 1 ? g.H - (p->Kr - 1) : g.H;
    rp.bnd_c = o->no_bndry_cross && p->Kc > 1 ? g.W - (p->Kc - 1) : g.W;
    rp.partials = part; rp.st = sts; rp.vstate = vstate ? 1 : 0;
    cp.g = g; cp.ph = pl.ph; cp.twH = twH; cp.twW = twW; cp.F = F; cp.Dh = Dh; cp.Sh = Sh;
    cp.grd = p->grd; cp.mu = p->mu; cp.wgrd = p->wgrd; cp.Psum = Psum; cp.st = sts;
    cp.E = Erows; cp.Kr = p->Kr;
    // The plain convolution solves write only their correction to the row
    // spectra of Y - U; the row pass adds Y - U itself (it holds both), so
    // the column pass reads each map's tile once instead of twice.  Not for
    // the masked (AMS) problems: there X = (Y - U) + correction, with Y - U
    // exact and the correction computed from its rounded spectra, doubles
    // the functional's rounding error (float32 emulation at 512 x 512,
    // 100 maps, 25 iterations: 7e-7 -> 1.2e-6 relative; unmasked problems:
    // 3e-7 -> 2e-7 to 4e-7).
    cp.delta = rp.delta =
        (col_mode == COL_SOLVE_C8 || col_mode == COL_SOLVE_C16) && p->mask == nullptr;
    fp.max_iter = o->max_iter;
    fp.auto_rho = o->auto_rho; fp.period = std::max(1, o->auto_rho_period);
    fp.auto_scaling = o->auto_scaling; fp.std_residuals = o->std_residuals;
    fp.rho_scaling = o->rho_scaling; fp.rsdl_ratio = o->rsdl_ratio;
    fp.abs_tol = o->abs_tol; fp.rel_tol = o->rel_tol;
    fp.nelem = (double)g.M * g.H * g.W;
    fp.xi = xi; fp.itstat = o->record_itstat ? it : nullptr; fp.ndone = ndone;
    // Without a stopping tolerance only a non-finite residual can end the
    // solve early; the host then never waits on the device mid-solve.
    can_stop = o->rel_tol > 0.f || o->abs_tol > 0.f;
    finished = o->max_iter <= 0;
    if (o->warm_start) {
      // The last iteration of the earlier solve may have changed rho; its
      // fix-up of the row spectra (Y - U / rsf) did not run because that
      // solve had finished.  Run it now (a no-op when rho did not change).
      if ((st = launch_row<ROW_FIXUP>(pl, rp, g.B, s))) return st;
    }
    if (tune && !o->warm_start && autotune_enabled() && o->max_iter > 0) {
      if ((st = tune_col())) return st;
    }
    return SC_OK;
  }

  // The starting iterates and their row spectra.
  int init_iterates() {
    const Geom& g = pl.g;
    const size_t real_all = (size_t)g.B * g.M * g.H * g.W;
    if (p->U0) {
      // start from the given iterates: U from U0, Y as given, F = rowFFT(Y - U)
      CU_TRY(cudaMemcpyAsync(U, p->U0, sizeof(float) * real_all, cudaMemcpyDeviceToDevice, s));
      CU_TRY(cudaMemsetAsync(F, 0, sizeof(float2) * (size_t)g.B * g.M * g.H * g.Wp, s));
      RowParams r = {};
      r.g = g; r.pw = pl.pw; r.twW = twW; r.F = F; r.Y = p->Y; r.U = U;
      int st = launch_row<ROW_FWD_YU>(pl, r, g.B, s);
      if (st) return st;
    } else {
      CU_TRY(cudaMemsetAsync(p->Y, 0, sizeof(float) * real_all, s));
      CU_TRY(cudaMemsetAsync(U, 0, sizeof(float) * real_all, s));
      CU_TRY(cudaMemsetAsync(F, 0, sizeof(float2) * (size_t)g.B * g.M * g.H * g.Wp, s));
    }
    return SC_OK;
  }

  // The column pass of the iteration at cluster size G, column radix rm,
  // tiles of tw columns and tail split G2 (0: the tuned choice, else the
  // model at the default radix and tile; G2 < 0: the tuned split).
  int launch_iter_col(int G, int rm = 0, int tw = 0, int G2 = -1) {
    const int B = pl.g.B;
    if (G <= 0) G = force_G;
    switch (col_mode) {
      case COL_SOLVE_W: return launch_col<COL_SOLVE_W>(pl, cp, B, s, G, rm, tw, G2);
      case COL_SOLVE: return launch_col<COL_SOLVE>(pl, cp, B, s, G, rm, tw, G2);
      case COL_SOLVE_C8: return launch_col<COL_SOLVE_C8>(pl, cp, B, s, G, rm, tw, G2);
      case COL_SOLVE_C16: return launch_col<COL_SOLVE_C16>(pl, cp, B, s, G, rm, tw, G2);
      case COL_SOLVE_G16: return launch_col<COL_SOLVE_G16>(pl, cp, B, s, G, rm, tw, G2);
      default: return launch_col<COL_SOLVE_P>(pl, cp, B, s, G, rm, tw, G2);
    }
  }
  // The iteration's column kernel with radix rm and tiles of tw columns
  // (nullptr when that variant is not compiled for the length).
  const void* iter_col_fn(int rm, int tw) const {
    const int H = pl.g.H;
    switch (col_mode) {
      case COL_SOLVE_W: return (const void*)col_fn_variant<COL_SOLVE_W>(H, rm, tw);
      case COL_SOLVE: return (const void*)col_fn_variant<COL_SOLVE>(H, rm, tw);
      case COL_SOLVE_C8: return (const void*)col_fn_variant<COL_SOLVE_C8>(H, rm, tw);
      case COL_SOLVE_C16: return (const void*)col_fn_variant<COL_SOLVE_C16>(H, rm, tw);
      case COL_SOLVE_G16: return (const void*)col_fn_variant<COL_SOLVE_G16>(H, rm, tw);
      default: return (const void*)col_fn_variant<COL_SOLVE_P>(H, rm, tw);
    }
  }

  // Autotuner of the column pass: the first solve of a shape in a process
  // times the iteration's column pass for every variant the length has
  // compiled: the column plan (the default radix, and radix 8 where the
  // default is 16: twice the threads per column, half the rows per thread),
  // the tile width (4 columns, or 2 for the convolution solves at lengths
  // from 512: half the threads and shared memory per CTA, twice the tiles)
  // and every cluster size the device can hold with it (kClusterSizes, at
  // most M); two rounds, the faster time of each kept, on the freshly
  // initialised state.  For one image it then times the fastest with the
  // tiles of a partly filled last round of clusters split off into a second
  // launch with larger clusters (TunedG::G2), and keeps the split where it
  // is faster by more than 1 %.  It keeps the fastest (radix, tile, cluster
  // size, split) for later launches of that shape and initialises the
  // iterates again (the trials overwrite the spectra).  It waits for the
  // device once, at that first set-up.
  int tune_col() {
    const Geom& g = pl.g;
    const int rdef = col_radix(g.H);
    const void* fn = iter_col_fn(rdef, SC_COL_TILE);
    int G0 = 0;
    if (forced_cluster(g.M) > 0 || tuned_size(fn, g, &G0)) return SC_OK;
    int st;
    struct Cand { int rm, tw, G; float ms; };
    std::vector<Cand> cand;
    for (int k = 0; k < 2; ++k) {
      const int rm = k ? 8 : rdef;
      if (k && rdef == 8) continue;
      for (int tw : {SC_COL_TILE, 2}) {
        const void* f = iter_col_fn(rm, tw);
        if (!f) continue;
        const ColShape sh = col_shape(g.H, rm, tw);
        if ((st = prepare_fn(f, true))) return st;
        const size_t smem = col_smem_bytes(col_mode, sh.hlen, tw);
        for (int G : kClusterSizes) {
          int n = 0;
          if (G > g.M) continue;
          if ((st = resident_clusters(f, sh.NT, smem, G, &n))) return st;
          if (n >= 1) cand.push_back({rm, tw, G, 1e30f});
        }
      }
    }
    const int nc = (int)cand.size();
    if (nc < 2) return SC_OK;  // nothing to choose
    cudaEvent_t e0, e1;
    CU_TRY(cudaEventCreate(&e0));
    CU_TRY(cudaEventCreate(&e1));
    st = SC_OK;
    for (int round = 0; round < 2 && !st; ++round) {
      for (int i = 0; i < nc && !st; ++i) {
        float ms = 0.f;
        if (cudaEventRecord(e0, s) != cudaSuccess) { st = SC_ERR_CUDA; break; }
        st = launch_iter_col(cand[i].G, cand[i].rm, cand[i].tw, 0);
        if (!st && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
            cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
          cand[i].ms = std::min(cand[i].ms, ms);
      }
    }
    int bi = 0;
    for (int i = 1; i < nc && !st; ++i)
      if (cand[i].ms < cand[bi].ms) bi = i;
    // the tail split of the fastest
    int best_G2 = 0;
    float best_ms = cand[bi].ms;
    std::vector<std::pair<int, float>> splits;
    for (int G2 : kClusterSizes) {
      if (st || g.B != 1 || G2 <= cand[bi].G || G2 > g.M) continue;
      float t2 = 1e30f;
      for (int round = 0; round < 2 && !st; ++round) {
        float ms = 0.f;
        if (cudaEventRecord(e0, s) != cudaSuccess) { st = SC_ERR_CUDA; break; }
        st = launch_iter_col(cand[bi].G, cand[bi].rm, cand[bi].tw, G2);
        if (!st && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
            cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
          t2 = std::min(t2, ms);
      }
      splits.push_back({G2, t2});
      if (t2 < 0.99f * best_ms) {
        best_ms = t2;
        best_G2 = G2;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if (autotune_verbose()) {
      fprintf(stderr, "sporco_b200 autotune: column pass %dx%d M=%d:", g.H, g.W, g.M);
      for (int i = 0; i < nc; ++i)
        fprintf(stderr, " r%d/t%d/G=%d %.3f ms", cand[i].rm, cand[i].tw, cand[i].G, cand[i].ms);
      for (const auto& sp : splits) fprintf(stderr, " split G2=%d %.3f ms", sp.first, sp.second);
      fprintf(stderr, " -> r%d/t%d/G=%d", cand[bi].rm, cand[bi].tw, cand[bi].G);
      if (best_G2 > 0) fprintf(stderr, " split G2=%d", best_G2);
      fprintf(stderr, "\n");
    }
    int dev = 0;
    CU_TRY(cudaGetDevice(&dev));
    {
      // a shape tuned meanwhile by another thread keeps its first answer
      std::lock_guard<std::mutex> lock(g_cache_mu);
      bool known = false;
      for (const TunedG& e : g_tuned)
        known = known || (e.dev == dev && e.fn == fn && e.H == g.H && e.W == g.W && e.M == g.M);
      if (!known)
        g_tuned.push_back(
            {dev, fn, g.H, g.W, g.M, cand[bi].G, cand[bi].rm, cand[bi].tw, best_G2});
    }
    return init_iterates();
  }

  // Iterations to launch before the next poll.
  int chunk() const {
    int c = o->max_iter - done_iters;
    if (o->check_every > 0) c = std::min(c, o->check_every);
    return c;
  }

  // Launch n ADMM iterations; timed(kind, launch) wraps every launch.
  template <typename Timed>
  int launch(int n, Timed&& timed) {
    const int B = pl.g.B;
    int st;
    for (int i = 0; i < n; ++i) {
      if ((st = timed(0, [&] {
             return launch_iter_col(0);
           })))
        return st;
      if ((st = timed(1, [&] {
             return vstate ? launch_row<ROW_ITER>(pl, rp, B, s)
                           : launch_row<ROW_ITER_YU>(pl, rp, B, s);
           })))
        return st;
      if ((st = timed(2, [&]() -> int {
             cudaLaunchConfig_t cfg = {};
             cfg.gridDim = dim3(B);
             cfg.blockDim = dim3(256);
             cfg.stream = s;
             cudaLaunchAttribute attr[1];
             set_pdl(&attr[0]);
             cfg.attrs = attr;
             cfg.numAttrs = pdl_enabled() ? 1 : 0;
             CU_TRY(cudaLaunchKernelEx(&cfg, finalize_kernel, (const double*)part,
                                       pl.row_nblk, sts, fp));
             ++g_launches;
             return o->record_itstat ? objective() : SC_OK;
           })))
        return st;
      if (o->auto_rho) {
        if ((st = timed(3, [&] { return launch_row<ROW_FIXUP>(pl, rp, B, s); }))) return st;
      }
    }
    done_iters += n;
    if (done_iters >= o->max_iter) finished = true;
    return SC_OK;
  }

  // Wait for the launched iterations and stop when every image is finished.
  // Between chunks: with a stopping test, wait for the chunk and read the
  // "finished" counter; without one, wait only for the chunk before (one
  // chunk stays queued, the device never idles).  Either way a cancellation
  // (sc_cancel) seen here stops the launches.
  int poll() {
    if (finished) return SC_OK;
    if (can_stop) {
      int nd = 0;
      CU_TRY(cudaMemcpyAsync(&nd, ndone, sizeof(int), cudaMemcpyDeviceToHost, s));
      CU_TRY(cudaStreamSynchronize(s));
      if (nd >= pl.g.B) finished = true;
    } else {
      for (int i = 0; i < 2; ++i)
        if (!pace[i]) CU_TRY(cudaEventCreateWithFlags(&pace[i], cudaEventDisableTiming));
      CU_TRY(cudaEventRecord(pace[nchunk & 1], s));
      if (nchunk > 0) CU_TRY(cudaEventSynchronize(pace[(nchunk - 1) & 1]));
      ++nchunk;
    }
    if (g_cancel_gen.load() != gen0) {
      cancelled = true;
      finished = true;
    }
    return SC_OK;
  }

  Solve() = default;
  Solve(const Solve&) = delete;  // owns its pacing events
  Solve& operator=(const Solve&) = delete;
  ~Solve() {
    for (int i = 0; i < 2; ++i)
      if (pace[i]) cudaEventDestroy(pace[i]);
  }

  // The functional at Y of the iteration just completed into the statistics
  // (record_itstat): Y from the state, its 2-D spectrum, then the fidelity,
  // gradient and L1 sums (cbpdn.cu:438-517).
  int objective() {
    const Geom& g = pl.g;
    unsigned char* ws = (unsigned char*)wsbase;
    float2* Yh = (float2*)(ws + pl.off_objspec);
    double* pspec = (double*)(ws + pl.off_objpart);
    double* pl1 = pspec + 2 * SC_OBJ_BLOCKS * g.B;
    int st;
    if (vstate && (st = state_yu(p->Y, nullptr))) return st;
    RowParams r = {};
    r.g = g; r.pw = pl.pw; r.twW = twW; r.F = Yh; r.src = p->Y;
    if ((st = launch_row<ROW_FWD_REAL>(pl, r, g.B, s))) return st;
    ColParams c = {};
    c.g = g; c.ph = pl.ph; c.twH = twH; c.twW = twW; c.F = Yh;
    if ((st = launch_col<COL_FWD>(pl, c, g.B, s))) return st;
    const dim3 grid(SC_OBJ_BLOCKS, g.B);
    objective_spec_kernel<<<grid, 256, 0, s>>>(Yh, Dh, Sh, g, p->grd, p->wgrd, twH, twW, pspec);
    objective_l1_kernel<<<grid, 256, 0, s>>>(p->Y, g, p->l1_kind, p->l1_scalar, p->l1w, pl1);
    objective_final_kernel<<<(g.B + 127) / 128, 128, 0, s>>>(
        pspec, pl1, SC_OBJ_BLOCKS, sts, p->lmbda, 1.0 / ((double)g.H * g.W),
        p->grd ? p->mu : 0.f, it, o->max_iter, g.B);
    CU_TRY(cudaGetLastError());
    g_launches += 3;
    return SC_OK;
  }

  // Y and U from the state V into y and u (u may be NULL).
  // Y and U from the state V (the solver's own, or v)
  int state_yu(float* y, float* u, const float* v = nullptr) {
    const Geom& g = pl.g;
    const size_t n = (size_t)g.M * g.H * g.W;
    dim3 grid((unsigned)std::min<size_t>((n + 255) / 256, 1024), g.B);
    state_yu_kernel<<<grid, 256, 0, s>>>(v ? v : U, y, u, sts, p->lmbda, g.M, g.H, g.W,
                                         p->l1_kind,
                                         p->l1_scalar, p->l1w, p->mask, rp.nonneg, rp.bnd_r,
                                         rp.bnd_c);
    CU_TRY(cudaGetLastError());
    ++g_launches;
    return SC_OK;
  }

  // trace steps without finalize (trace_state_kernel)
  int trace_state() {
    trace_state_kernel<<<(pl.g.B + 127) / 128, 128, 0, s>>>(sts, pl.g.B);
    CU_TRY(cudaGetLastError());
    ++g_launches;
    return SC_OK;
  }

  int export_u() {
    if (vstate) return state_yu(p->Y, p->U_out);
    if (!p->U_out) return SC_OK;
    const size_t per = (size_t)pl.g.M * pl.g.H * pl.g.W, n = per * pl.g.B;
    export_u_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s>>>(
        U, p->U_out, sts, per, n);
    CU_TRY(cudaGetLastError());
    ++g_launches;
    return SC_OK;
  }

  int result(sc_result* res) {
    int st = export_u();
    if (st) return st;
    if (cancelled) {
      CU_TRY(cudaStreamSynchronize(s));
      return set_status(SC_ERR_CANCELLED, "solve cancelled (sc_cancel) after %d iterations",
                        done_iters);
    }
    if (!res) return SC_OK;
    const int B = pl.g.B;
    ImgState h0;
    CU_TRY(cudaMemcpyAsync(&h0, sts, sizeof(ImgState), cudaMemcpyDeviceToHost, s));
    CU_TRY(cudaStreamSynchronize(s));
    res->iterations = h0.k - h0.k0;
    res->rho = h0.rho;
    res->r = h0.r;
    res->s = h0.s;
    if (B > 1) {
      std::vector<ImgState> hs(B);
      CU_TRY(cudaMemcpy(hs.data(), sts, sizeof(ImgState) * B, cudaMemcpyDeviceToHost));
      for (auto& x : hs) res->iterations = std::max(res->iterations, x.k - x.k0);
      for (auto& x : hs)
        if (x.status) return set_status(x.status, "non-finite residual");
    }
    if (h0.status) return set_status(h0.status, "non-finite residual");
    return SC_OK;
  }
};

extern "C" int sc_cbpdn_solve(const sc_problem* p, const sc_options* o, void* workspace,
                              size_t workspace_bytes, sc_result* res, void* stream) {
  set_status(SC_OK, nullptr);
  (void)cudaGetLastError();  // do not report an earlier call's error as ours
  Solve sv;
  cudaStream_t s = (cudaStream_t)stream;
  int st = sv.setup(p, o, workspace, workspace_bytes, s);
  if (st) return st;

  // Per-kernel event timing (profile mode only); events come from a
  // grow-only pool so that profiling adds no per-launch host allocation.
  struct EvRec { cudaEvent_t a, b; int kind; };
  static thread_local std::vector<cudaEvent_t> ev_pool;
  std::vector<EvRec> evs;
  size_t ev_next = 0;
  auto get_ev = [&](cudaEvent_t* e) -> int {
    if (ev_next == ev_pool.size()) {
      cudaEvent_t x;
      CU_TRY(cudaEventCreate(&x));
      ev_pool.push_back(x);
    }
    *e = ev_pool[ev_next++];
    return SC_OK;
  };
  auto timed = [&](int kind, auto&& launch) -> int {
    if (!o->profile) return launch();
    EvRec e;
    e.kind = kind;
    int r = get_ev(&e.a);
    if (!r) r = get_ev(&e.b);
    if (r) return r;
    CU_TRY(cudaEventRecord(e.a, s));
    r = launch();
    CU_TRY(cudaEventRecord(e.b, s));
    evs.push_back(e);
    return r;
  };
  while (!sv.finished) {
    if ((st = sv.launch(sv.chunk(), timed))) return st;
    if ((st = sv.poll())) return st;
  }
  if (o->profile) {
    CU_TRY(cudaStreamSynchronize(s));
    memset(&g_profile, 0, sizeof(g_profile));
    for (auto& e : evs) {
      float ms = 0.f;
      CU_TRY(cudaEventElapsedTime(&ms, e.a, e.b));
      g_profile.ms[e.kind] += ms;
      g_profile.count[e.kind] += 1;
    }
  }
  return sv.result(res);
}

extern "C" int sc_cbpdn_solve_batch(const sc_problem* probs, int nprob, const sc_options* o,
                                    void* const* workspaces, const size_t* workspace_bytes,
                                    sc_result* res, void* const* streams) {
  set_status(SC_OK, nullptr);
  (void)cudaGetLastError();
  if (!probs || nprob < 1 || !o || !workspaces || !workspace_bytes)
    return set_status(SC_ERR_INVALID, "invalid batch arguments");
  if (o->profile) return set_status(SC_ERR_INVALID, "profiling is per single solve");
  std::vector<Solve> sv(nprob);
  int st;
  for (int i = 0; i < nprob; ++i) {
    cudaStream_t s = streams ? (cudaStream_t)streams[i] : nullptr;
    if ((st = sv[i].setup(&probs[i], o, workspaces[i], workspace_bytes[i], s))) return st;
  }
  auto untimed = [](int, auto&& launch) -> int { return launch(); };
  for (;;) {
    bool any = false;
    for (auto& x : sv) {
      if (x.finished) continue;
      any = true;
      if ((st = x.launch(x.chunk(), untimed))) return st;
    }
    if (!any) break;
    for (auto& x : sv)
      if ((st = x.poll())) return st;
  }
  for (int i = 0; i < nprob; ++i)
    if ((st = sv[i].result(res ? &res[i] : nullptr))) return st;
  return SC_OK;
}

// ------------------------------------------------ unrolled solve + adjoint --
// Workspace of the unrolled solve: the solver's own workspace first, then
//   ckV      (nseg, B, M, H, W)  the state V = Y + U at the start of every segment
//   Yt, Ut   (B, M, H, W)        Y and U of a segment's start (its restart)
//   Vtr      (seg, B, M, H, W)   V after each step of the segment being reversed
//                                (Y of the step = its shrinkage)
//   Xtr      (seg, B, M, H, Wp)  x^ of each of those steps
//   gV       (B, M, H, W)        gradient w.r.t. V of the step being reversed
//   Fb       (B, M, H, Wp)       spectra of the reverse steps
//   gDh      (B, M, H, Wp), gSh (B, H, Wp)  gradient spectra, per image
//   gDr      (M, H, W)           dictionary gradient before the crop
struct Unrolled {
  sc_problem p;   // the caller's problem with the solver-owned fields cleared
  sc_options o;   // fixed rho, no stopping test, no statistics
  Plan pl;
  int K = 0, seg = 0, nseg = 0;
  size_t R = 0, C = 0;  // floats of a real array, complex entries of a spectrum array
  size_t ckV = 0, Yt = 0, Ut = 0, Vtr = 0, Xtr = 0, gV = 0, Fb = 0, gDh = 0, gSh = 0, gDr = 0;
  // convolution form (filters of at most 16 rows, compiled column lengths
  // below 512): the forward and the recomputation use the production
  // convolution solve, the reverse pass its convolution-form adjoint
  bool conv = false;
  int conv_mode = 0, trace_mode = 0, adj_mode = 0;
  size_t SCtr = 0, gE = 0;
  size_t total = 0;
};

// SPORCO_B200_ADJOINT=transform keeps the transform-solve adjoint for every
// problem (the form used before the convolution form; for comparisons).
static bool adjoint_transform_forced() {
  const char* e = getenv("SPORCO_B200_ADJOINT");
  return e && strcmp(e, "transform") == 0;
}

static int unrolled_plan(const sc_problem* p, const sc_options* o, int seg, Unrolled* u) {
  if (!p || !o) return set_status(SC_ERR_INVALID, "null problem or options");
  if (p->grd || p->mask || p->U0 || p->U_out)
    return set_status(SC_ERR_UNSUPPORTED,
                      "the unrolled solve is plain cbpdn (no gradient term, mask or warm start)");
  if (o->max_iter < 1) return set_status(SC_ERR_INVALID, "max_iter must be >= 1");
  if (seg < 1 || seg > o->max_iter)
    return set_status(SC_ERR_INVALID, "segment length %d outside 1..%d", seg, o->max_iter);
  u->p = *p;
  u->o = *o;
  u->o.rel_tol = 0.f;
  u->o.abs_tol = 0.f;
  u->o.auto_rho = 0;
  u->o.record_itstat = 0;
  u->o.check_every = 0;
  u->o.profile = 0;
  int st = plan_problem(&u->p, &u->o, &u->pl);
  if (st) return st;
  const Geom& g = u->pl.g;
  u->K = o->max_iter;
  u->seg = seg;
  u->nseg = (u->K + seg - 1) / seg;
  u->R = (size_t)g.B * g.M * g.H * g.W;
  u->C = (size_t)g.B * g.M * g.H * g.Wp;
  size_t off = u->pl.total;
  auto take = [&](size_t bytes) { size_t r = off; off = align256(off + bytes); return r; };
  u->ckV = take(sizeof(float) * u->R * u->nseg);
  u->Yt = take(sizeof(float) * u->R);
  u->Ut = take(sizeof(float) * u->R);
  u->Vtr = take(sizeof(float) * u->R * seg);
  u->Xtr = take(sizeof(float2) * u->C * seg);
  u->gV = take(sizeof(float) * u->R);
  u->Fb = take(sizeof(float2) * u->C);
  u->gDh = take(sizeof(float2) * u->C);
  u->gSh = take(sizeof(float2) * (size_t)g.B * g.H * g.Wp);
  u->gDr = take(sizeof(float) * (size_t)g.M * g.H * g.W);
  u->conv = !adjoint_transform_forced() && spec_col(g.H) && col_radix(g.H) == 8 &&
            p->Kr <= 16;
  if (u->conv) {
    const bool c8 = p->Kr <= 8;
    u->conv_mode = c8 ? COL_SOLVE_C8 : COL_SOLVE_C16;
    u->trace_mode = c8 ? COL_SOLVE_C8T : COL_SOLVE_C16T;
    u->adj_mode = c8 ? COL_ADJ_C8 : COL_ADJ_C16;
    u->SCtr = take(sizeof(float2) * (size_t)g.B * g.H * g.Wp * seg);
    u->gE = take(sizeof(float2) * (size_t)g.B * g.M * p->Kr * g.Wp);
  }
  u->total = off;
  return SC_OK;
}

// Cluster size of the unrolled forward and of its recomputation, which must
// sum the maps in the same order: the autotuned size of the production
// convolution solve for this shape (the forward tunes it), else the
// occupancy model of the trace kernel.
static int unrolled_cluster(const Unrolled& u, int* G) {
  const void* fc = u.conv_mode == COL_SOLVE_C8 ? (const void*)col_fn<COL_SOLVE_C8>(u.pl.g.H)
                                               : (const void*)col_fn<COL_SOLVE_C16>(u.pl.g.H);
  int rm = 0, tw = 0;
  if (tuned_size(fc, u.pl.g, G, &rm, &tw) && rm == col_radix(u.pl.g.H) && tw == SC_COL_TILE)
    return SC_OK;
  const void* fn = u.trace_mode == COL_SOLVE_C8T ? (const void*)col_fn<COL_SOLVE_C8T>(u.pl.g.H)
                                                 : (const void*)col_fn<COL_SOLVE_C16T>(u.pl.g.H);
  int st = prepare_fn(fn, true);
  if (st) return st;
  return cluster_size(fn, u.pl.col_NT, col_smem_bytes(u.trace_mode, u.pl.col_hlen), u.pl.g.M,
                      (long)u.pl.col_ntiles * u.pl.g.B, G);
}

extern "C" size_t sc_unrolled_workspace_size(const sc_problem* p, const sc_options* o, int seg) {
  Unrolled u;
  if (unrolled_plan(p, o, seg, &u)) return 0;
  return u.total;
}

static int unrolled_begin(const sc_problem* p, const sc_options* o, int seg, void* ws,
                          size_t bytes, Unrolled* u) {
  set_status(SC_OK, nullptr);
  (void)cudaGetLastError();
  int st = unrolled_plan(p, o, seg, u);
  if (st) return st;
  if (!ws || bytes < u->total)
    return set_status(SC_ERR_WORKSPACE, "workspace of %zu bytes needed", u->total);
  return SC_OK;
}

static auto untimed = [](int, auto&& launch) -> int { return launch(); };

extern "C" int sc_unrolled_forward(const sc_problem* p, const sc_options* o, int seg, void* ws,
                                   size_t bytes, void* stream) {
  Unrolled u;
  int st = unrolled_begin(p, o, seg, ws, bytes, &u);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* w = (unsigned char*)ws;
  Solve sv;
  sv.tune = false;  // forward and recomputation must use the same cluster sizes
  if ((st = sv.setup(&u.p, &u.o, ws, u.pl.total, s))) return st;
  // the recomputation's trace twins write the whole row spectra of X: the
  // forward does the same, so that both produce the same iterates
  sv.cp.delta = sv.rp.delta = 0;
  // the same column solve as the recomputation in the reverse pass, so that
  // both produce the same iterates: the production convolution solve (the
  // recomputation runs its trace-keeping twin) at a fixed cluster size, or
  // the transform solve
  if (u.conv) {
    sv.col_mode = u.conv_mode;
    // the first solve of a shape tunes the cluster size of the production
    // solve (the recomputation then uses the same size)
    if (autotune_enabled() && (st = sv.tune_col())) return st;
    if ((st = unrolled_cluster(u, &sv.force_G))) return st;
  } else {
    sv.col_mode = COL_SOLVE;
  }
  if (u.conv && u.seg == u.K) {
    // One segment (seg = K): the forward keeps the trace of every step that
    // the reverse pass needs (V, the row spectra of X and sc / rho), so the
    // backward recomputes nothing.  The trace-keeping kernels are the
    // recomputation's: the column pass's twin and the iteration's row pass
    // writing each step's V to a trace slot.
    float* Vtr = (float*)(w + u.Vtr);
    float2* Xtr = (float2*)(w + u.Xtr);
    float2* SCtr = (float2*)(w + u.SCtr);
    const Geom& g = u.pl.g;
    const size_t Cs = (size_t)g.B * g.H * g.Wp;
    if ((st = sv.trace_state())) return st;
    auto Vat = [&](int i) { return i == 0 ? sv.U : Vtr + u.R * (i - 1); };  // V_0 = 0
    for (int i = 0; i < u.K; ++i) {
      ColParams cf = sv.cp;
      cf.Xtr = Xtr + u.C * i;
      cf.SCtr = SCtr + Cs * i;
      st = u.trace_mode == COL_SOLVE_C8T ? launch_col<COL_SOLVE_C8T>(u.pl, cf, g.B, s, sv.force_G)
                                         : launch_col<COL_SOLVE_C16T>(u.pl, cf, g.B, s, sv.force_G);
      if (st) return st;
      RowParams rr = sv.rp;
      rr.U = Vat(i);
      rr.Vo = Vat(i + 1);
      if ((st = launch_row<ROW_ITER>(u.pl, rr, g.B, s))) return st;
    }
    return sv.state_yu(p->Y, (float*)(w + u.Ut), Vat(u.K));
  }
  for (int j = 0; j < u.nseg; ++j) {
    // the state V at the segment's start
    CU_TRY(cudaMemcpyAsync(w + u.ckV + sizeof(float) * u.R * j, sv.U, sizeof(float) * u.R,
                           cudaMemcpyDeviceToDevice, s));
    if ((st = sv.launch(std::min(u.seg, u.K - j * u.seg), untimed))) return st;
  }
  sc_result res;
  return sv.result(&res);
}

// gDh[0] <- sum over the images of gDh[b] (per: complex entries of one image)
__global__ void sum_images_kernel(float2* g, int B, size_t per) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < per;
       i += (size_t)gridDim.x * blockDim.x) {
    float2 a = g[i];
    for (int b = 1; b < B; ++b) {
      const float2 v = g[(size_t)b * per + i];
      a.x += v.x;
      a.y += v.y;
    }
    g[i] = a;
  }
}

// gD (M, Kr, Kc) <- the filter support of src (M, H, W)
__global__ void crop_kernel(const float* src, float* dst, int M, int H, int W, int Kr, int Kc) {
  const int n = M * Kr * Kc;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int m = i / (Kr * Kc), r = (i / Kc) % Kr, c = i % Kc;
    dst[i] = src[((size_t)m * H + r) * W + c];
  }
}

// Reverse pass.  Step k of the forward pass maps (Y_k, U_k) to (Y_k+1, U_k+1)
// through X_k = A^{-1}(D^T S + rho (Y_k - U_k)), V_k = a X_k + (1 - a) Y_k + U_k,
// Y_k+1 = soft(V_k), U_k+1 = V_k - Y_k+1.  Its reverse: gV_k from the
// gradients w.r.t. Y_k+1 and U_k+1 and the shrinkage mask (Y_k+1 != 0), then
// (COL_ADJ) Q_k = A^{-1} a gV_k with the dictionary and signal gradients, then
// (ROW_ADJ) the gradients w.r.t. Y_k and U_k, which give gV_k-1.  Segments are
// reversed last to first, each after recomputing its forward steps from its
// checkpoint with Y and x^ of every step kept.
extern "C" int sc_unrolled_backward(const sc_problem* p, const sc_options* o, int seg, void* ws,
                                    size_t bytes, const float* gY, float* gD, float* gS,
                                    void* stream) {
  Unrolled u;
  int st = unrolled_begin(p, o, seg, ws, bytes, &u);
  if (st) return st;
  if (!gY || !gD || !gS) return set_status(SC_ERR_INVALID, "null gradient pointer");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* w = (unsigned char*)ws;
  float* ckV = (float*)(w + u.ckV);
  float* Yt = (float*)(w + u.Yt);
  float* Ut = (float*)(w + u.Ut);
  float* Vtr = (float*)(w + u.Vtr);
  float2* Xtr = (float2*)(w + u.Xtr);
  float* gV = (float*)(w + u.gV);
  float2* Fb = (float2*)(w + u.Fb);
  float2* gDh = (float2*)(w + u.gDh);
  float2* gSh = (float2*)(w + u.gSh);
  float* gDr = (float*)(w + u.gDr);
  float2* SCtr = u.conv ? (float2*)(w + u.SCtr) : nullptr;
  float2* gE = u.conv ? (float2*)(w + u.gE) : nullptr;
  const Geom& g = u.pl.g;
  const Plan& pl = u.pl;
  const int B = g.B;
  const int Kr = u.p.Kr;
  const size_t Cs = (size_t)B * g.H * g.Wp;  // complex entries of one SC trace
  int G = 0;
  if (u.conv && (st = unrolled_cluster(u, &G))) return st;
  // one segment with the convolution form: the forward kept every step's
  // trace, nothing is recomputed
  const bool traced = u.conv && u.seg == u.K;
  // set-up writes zeros to the problem's Y: give it the restart's scratch
  u.p.Y = Yt;
  Solve sv;
  sv.tune = false;
  if ((st = sv.setup(&u.p, &u.o, ws, pl.total, s))) return st;
  sv.cp.delta = sv.rp.delta = 0;  // as in the forward
  if ((st = sv.trace_state())) return st;
  if (u.conv)
    CU_TRY(cudaMemsetAsync(gE, 0, sizeof(float2) * (size_t)B * g.M * Kr * g.Wp, s));
  else
    CU_TRY(cudaMemsetAsync(gDh, 0, sizeof(float2) * u.C, s));
  CU_TRY(cudaMemsetAsync(gSh, 0, sizeof(float2) * Cs, s));
  CU_TRY(cudaMemcpyAsync(gV, gY, sizeof(float) * u.R, cudaMemcpyDeviceToDevice, s));

  RowParams ra = sv.rp;
  ra.F = Fb; ra.gV = gV; ra.first = 1; ra.vmask = 1;
  ColParams ca = sv.cp;
  ca.F = Fb; ca.gDh = gDh; ca.gSh = gSh; ca.Xtr = nullptr; ca.gE = gE;
  for (int j = u.nseg - 1; j >= 0; --j) {
    const int n = std::min(u.seg, u.K - j * u.seg);
    // V of step i of this segment: i = 0 is the checkpoint
    auto Vat = [&](int i) { return i == 0 ? ckV + u.R * j : Vtr + u.R * (i - 1); };
    // recompute the segment: the row spectra of Y - U at its start (from
    // the Y and U of the checkpoint's V, transformed as the iteration does)
    if (!traced) {
      if ((st = sv.state_yu(Yt, Ut, Vat(0)))) return st;
      RowParams rf = sv.rp;
      rf.Y = Yt;
      rf.U = Ut;
      if ((st = launch_row<ROW_FWD_YU>(pl, rf, B, s))) return st;
    }
    for (int i = 0; i < n && !traced; ++i) {
      ColParams cf = sv.cp;
      cf.Xtr = Xtr + u.C * i;
      if (u.conv) {
        cf.SCtr = SCtr + Cs * i;
        st = u.trace_mode == COL_SOLVE_C8T ? launch_col<COL_SOLVE_C8T>(pl, cf, B, s, G)
                                           : launch_col<COL_SOLVE_C16T>(pl, cf, B, s, G);
      } else {
        st = launch_col<COL_SOLVE_X>(pl, cf, B, s);
      }
      if (st) return st;
      RowParams rr = sv.rp;
      rr.U = Vat(i);
      rr.Vo = Vat(i + 1);
      if ((st = launch_row<ROW_ITER>(pl, rr, B, s))) return st;
    }
    // reverse it
    ra.Ymask = Vat(n);
    if ((st = launch_row<ROW_ADJ>(pl, ra, B, s))) return st;
    ra.first = 0;
    for (int i = n - 1; i >= 0; --i) {
      ca.Xh = Xtr + u.C * i;
      if (u.conv) {
        ca.SCtr = SCtr + Cs * i;
        st = u.adj_mode == COL_ADJ_C8 ? launch_col<COL_ADJ_C8>(pl, ca, B, s)
                                      : launch_col<COL_ADJ_C16>(pl, ca, B, s);
      } else {
        st = launch_col<COL_ADJ>(pl, ca, B, s);
      }
      if (st) return st;
      if (i > 0) {
        ra.Ymask = Vat(i);
        if ((st = launch_row<ROW_ADJ>(pl, ra, B, s))) return st;
      }
    }
  }
  // dictionary gradient: sum over the images, inverse FFT, crop to the filters
  if (u.conv) {
    // gE holds, per filter row t, H^2 IFFTcol(gD^)(t) in the row-spectral
    // domain: the inverse row transform with 1 / (H^2 W) gives the spatial
    // gradient at the filter rows
    const size_t per = (size_t)g.M * Kr * g.Wp;
    sum_images_kernel<<<(unsigned)std::min<size_t>((per + 255) / 256, 4096), 256, 0, s>>>(gE, B,
                                                                                         per);
    CU_TRY(cudaGetLastError());
    ++g_launches;
    RowParams ri = sv.rp;
    ri.g.B = 1; ri.g.H = Kr; ri.F = gE; ri.dst = gDr;
    ri.invN = (float)(1.0 / ((double)g.H * g.H * g.W));
    if ((st = launch_row<ROW_INV_REAL>(pl, ri, 1, s))) return st;
    const int nk = g.M * Kr * u.p.Kc;
    crop_kernel<<<(nk + 255) / 256, 256, 0, s>>>(gDr, gD, g.M, Kr, g.W, Kr, u.p.Kc);
    CU_TRY(cudaGetLastError());
    ++g_launches;
  } else {
    const size_t per = (size_t)g.M * g.H * g.Wp;
    sum_images_kernel<<<(unsigned)std::min<size_t>((per + 255) / 256, 4096), 256, 0, s>>>(gDh, B,
                                                                                         per);
    CU_TRY(cudaGetLastError());
    ++g_launches;
    ColParams ci = sv.cp;
    ci.g.B = 1; ci.F = gDh;
    if ((st = launch_col<COL_INV>(pl, ci, 1, s))) return st;
    RowParams ri = sv.rp;
    ri.g.B = 1; ri.F = gDh; ri.dst = gDr;
    if ((st = launch_row<ROW_INV_REAL>(pl, ri, 1, s))) return st;
    const int nk = g.M * u.p.Kr * u.p.Kc;
    crop_kernel<<<(nk + 255) / 256, 256, 0, s>>>(gDr, gD, g.M, g.H, g.W, u.p.Kr, u.p.Kc);
    CU_TRY(cudaGetLastError());
    ++g_launches;
  }
  // signal gradient
  {
    ColParams ci = sv.cp;
    ci.g.M = 1; ci.F = gSh;
    if ((st = launch_col<COL_INV>(pl, ci, B, s))) return st;
    RowParams ri = sv.rp;
    ri.g.M = 1; ri.F = gSh; ri.dst = gS;
    if ((st = launch_row<ROW_INV_REAL>(pl, ri, B, s))) return st;
  }
  return SC_OK;
}

extern "C" int sc_read_state(const sc_problem* p, const sc_options* o, const void* workspace,
                             int* iterations, double* rho, double* itstat, void* stream) {
  Plan pl;
  int st = plan_problem(p, o, &pl);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned char* ws = (const unsigned char*)workspace;
  std::vector<ImgState> hs(pl.g.B);
  CU_TRY(cudaMemcpyAsync(hs.data(), ws + pl.off_st, sizeof(ImgState) * pl.g.B,
                         cudaMemcpyDeviceToHost, s));
  if (itstat && o->record_itstat)
    CU_TRY(cudaMemcpyAsync(itstat, ws + pl.off_it,
                           sizeof(double) * SC_ITSTAT_FIELDS * (size_t)std::max(1, o->max_iter) *
                               pl.g.B,
                           cudaMemcpyDeviceToHost, s));
  CU_TRY(cudaStreamSynchronize(s));
  for (int b = 0; b < pl.g.B; ++b) {
    if (iterations) iterations[b] = hs[b].k - hs[b].k0;
    if (rho) rho[b] = hs[b].rho;
  }
  return SC_OK;
}

// --------------------------------------------------------------- rfft2 tools --
// Twiddle tables of the FFT tool entry points, kept per (device, W, H) for
// the life of the process (a handful of sizes in practice).
struct TwEntry {
  int dev, W, H;
  float2* tw;
};
static std::vector<TwEntry> g_tw_cache;

static int tool_twiddles(int W, int H, cudaStream_t s, float2** out) {
  int dev = 0;
  CU_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (auto& e : g_tw_cache)
    if (e.dev == dev && e.W == W && e.H == H) {
      *out = e.tw;
      return SC_OK;
    }
  float2* tw = nullptr;
  CU_TRY(cudaMalloc((void**)&tw, sizeof(float2) * (W + H)));
  twiddle_kernel<<<(W + 255) / 256, 256, 0, s>>>(tw, W);
  twiddle_kernel<<<(H + 255) / 256, 256, 0, s>>>(tw + W, H);
  CU_TRY(cudaGetLastError());
  // other threads may use the table at once, from other streams
  CU_TRY(cudaStreamSynchronize(s));
  g_tw_cache.push_back({dev, W, H, tw});
  *out = tw;
  return SC_OK;
}

extern "C" int sc_rfft2(const float* x, void* xf, int count, int H, int W, void* stream) {
  set_status(SC_OK, nullptr);
  (void)cudaGetLastError();
  Plan pl;
  int st = plan_geometry(count, 1, H, W, &pl);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  pl.g.Wp = pl.g.Wf;  // dense numpy layout
  float2* tw = nullptr;
  if ((st = tool_twiddles(W, H, s, &tw))) return st;
  RowParams rp = {};
  rp.g = pl.g; rp.pw = pl.pw; rp.twW = tw; rp.F = (float2*)xf; rp.src = x;
  if ((st = launch_row<ROW_FWD_REAL>(pl, rp, count, s))) return st;
  ColParams cp = {};
  cp.g = pl.g; cp.ph = pl.ph; cp.twH = tw + W; cp.twW = tw; cp.F = (float2*)xf;
  if ((st = launch_col<COL_FWD>(pl, cp, count, s))) return st;
  return SC_OK;
}

extern "C" int sc_irfft2(const void* xf, float* x, int count, int H, int W, void* stream) {
  set_status(SC_OK, nullptr);
  (void)cudaGetLastError();
  Plan pl;
  int st = plan_geometry(count, 1, H, W, &pl);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  pl.g.Wp = pl.g.Wf;
  float2* tw = nullptr;
  float2* tmp = nullptr;
  const size_t nspec = (size_t)count * H * pl.g.Wf;
  if ((st = tool_twiddles(W, H, s, &tw))) return st;
  CU_TRY(cudaMallocAsync((void**)&tmp, sizeof(float2) * nspec, s));
  CU_TRY(cudaMemcpyAsync(tmp, xf, sizeof(float2) * nspec, cudaMemcpyDeviceToDevice, s));
  ColParams cp = {};
  cp.g = pl.g; cp.ph = pl.ph; cp.twH = tw + W; cp.twW = tw; cp.F = tmp;
  if ((st = launch_col<COL_INV>(pl, cp, count, s))) return st;
  RowParams rp = {};
  rp.g = pl.g; rp.pw = pl.pw; rp.twW = tw; rp.F = tmp; rp.dst = x;
  rp.invN = (float)(1.0 / ((double)H * W));
  if ((st = launch_row<ROW_INV_REAL>(pl, rp, count, s))) return st;
  CU_TRY(cudaFreeAsync(tmp, s));
  return SC_OK;
}

// ------------------------------------------------- allocation-free rfft2 --
// sc_rfft2 takes its scratch (the two twiddle tables) from the stream-ordered
// allocator.  sc_rfft2_noalloc is the same transform with that scratch in a
// file-scope device array instead, for callers that must not allocate device
// memory.  The array is SC_NOALLOC_TWIDDLES complex entries (64 KiB) and
// holds the W + H twiddles of one call; every GPU that loads this library
// keeps it until the process exits.  All calls share it: each call rewrites
// the entries it uses before reading them (nothing has to start at zero),
// and calls that overlap on the GPU (e.g. on two streams) race on it.
#define SC_NOALLOC_TWIDDLES 8192
#define SC_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) float2 sc_noalloc_tw[SC_NOALLOC_TWIDDLES];
// Device address of sc_noalloc_tw per device (the host-side symbol is only a
// stand-in for it), looked up once per device by the first call there, under
// g_cache_mu.
static float2* g_noalloc_tw[SC_NOALLOC_MAX_DEVICES] = {};

extern "C" int sc_rfft2_noalloc(const float* x, void* xf, int count, int H, int W, void* stream) {
  set_status(SC_OK, nullptr);
  (void)cudaGetLastError();
  if (!x || !xf) return set_status(SC_ERR_INVALID, "null pointer");
  if (count < 1 || H < 1 || W < 1)
    return set_status(SC_ERR_INVALID, "sizes must be positive (count=%d H=%d W=%d)", count, H, W);
  if (H + W > SC_NOALLOC_TWIDDLES)
    return set_status(SC_ERR_UNSUPPORTED,
                      "H + W = %d twiddles exceed the %d the static scratch holds", H + W,
                      SC_NOALLOC_TWIDDLES);
  Plan pl;
  int st = plan_geometry(count, 1, H, W, &pl);
  if (st) return st;
  int dev = 0;
  CU_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= SC_NOALLOC_MAX_DEVICES)
    return set_status(SC_ERR_UNSUPPORTED, "device %d beyond the %d this entry point tracks", dev,
                      SC_NOALLOC_MAX_DEVICES);
  float2* tw = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    if (!g_noalloc_tw[dev]) {
      void* addr = nullptr;
      CU_TRY(cudaGetSymbolAddress(&addr, sc_noalloc_tw));
      g_noalloc_tw[dev] = (float2*)addr;
    }
    tw = g_noalloc_tw[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  pl.g.Wp = pl.g.Wf;  // dense numpy layout
  twiddle_kernel<<<(W + 255) / 256, 256, 0, s>>>(tw, W);
  twiddle_kernel<<<(H + 255) / 256, 256, 0, s>>>(tw + W, H);
  CU_TRY(cudaGetLastError());
  RowParams rp = {};
  rp.g = pl.g; rp.pw = pl.pw; rp.twW = tw; rp.F = (float2*)xf; rp.src = x;
  rp.gsz = pl.rowg_g;
  rp.nblk = pl.row_nblk;
  // the same one-time opt-in to the device's shared-memory maximum as every
  // other launch of these kernels (never lowered per call)
  const RowFn rfn = row_fn<ROW_FWD_REAL>(0);  // the runtime-plan instantiations
  const ColFn cfn = col_fn<COL_FWD>(0);
  if ((st = prepare_fn((const void*)rfn, false))) return st;
  if ((st = prepare_fn((const void*)cfn, false))) return st;
  {
    void* args[] = {&rp};
    CU_TRY(cudaLaunchKernel((const void*)rfn, dim3(rp.nblk, count),
                            dim3((SC_ROW_THREADS / rp.gsz) * rp.gsz), args, pl.rowg_smem, s));
  }
  ColParams cp = {};
  cp.g = pl.g; cp.ph = pl.ph; cp.twH = tw + W; cp.twW = tw; cp.F = (float2*)xf;
  cp.gsz = pl.colg_g;
  cp.Hs = pl.Hs;
  cp.G = 1;
  {
    void* args[] = {&cp};
    CU_TRY(cudaLaunchKernel((const void*)cfn, dim3(1, pl.col_ntiles, count), dim3(pl.colg_NT),
                            args, pl.colg_smem, s));
  }
  g_launches += 4;
  return SC_OK;
}
