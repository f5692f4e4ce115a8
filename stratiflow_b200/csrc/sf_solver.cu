// C-ABI of the B200 IMEX-RK engine: solver set-up, state transfer, and the
// step sequencer (one CUDA graph per step, replayed).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/stratiflow_b200.h"
#include "sf_internal.cuh"

using namespace sf;

static thread_local std::string g_err;

// used by the other translation units of the library
void sf_set_error_message(const std::string& msg) { g_err = msg; }

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e__ = (call);                                                                 \
    if (e__ != cudaSuccess)                                                                   \
      return fail(SF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e__));             \
  } while (0)

struct sf_solver {
  Geo g{};
  int device = 0;
  cudaStream_t st = nullptr;
  double L1 = 0, L2 = 0, L3 = 0, Re = 0, Pr = 0, dt = 0;
  float h[3] = {0, 0, 0};
  // device buffers
  float2* S[2] = {nullptr, nullptr};
  float2 *rold = nullptr, *rnl = nullptr, *qbuf = nullptr, *mixin = nullptr, *mixout = nullptr;
  float* base = nullptr;
  float *zc = nullptr, *fa = nullptr, *fc = nullptr, *inv_den = nullptr;
  float *kx = nullptr, *ky = nullptr, *Ri = nullptr, *Ubar = nullptr, *dBdz = nullptr;
  double *bands = nullptr, *kxd = nullptr, *kyd = nullptr, *red = nullptr;
  float2* tw = nullptr;
  float2* stage_ref = nullptr;   // one field in the reference layout
  float2* adir = nullptr;        // adjoint step: the direct state of the substep
  float2* amix = nullptr;        // 3D adjoint step: 12 y-transformed fields
  std::vector<float> hRi;
  std::vector<double> zN, zfN;   // grid (for inspection)
  int cur = 0;                   // index of the current state buffer
  bool base_set = false;
  int tlm = 0;                   // tangent-linear batch (sf_set_tangent)
  int xslabs = 0;                // slabs per x-pass block (sf_set_xpass_slabs)
  XYAux xy{};                    // side streams of the banded 3D x-y pass
  int xy_bands = 1;              // level bands of the 3D x-y pass (sf_set_xy_bands)
  int zchunks = 0;               // z chunks per z-solve block (sf_set_z_chunks)
  int xgroups = 0;               // lane groups per x-pass block (sf_set_xpass_groups)
  int xkernel = 1;               // 3D nonlinear x pass: 1 level-marching, 0 slab blocks (sf_set_xpass_kernel)
  int zkernel = 2;               // z pass: 2 k_z_step_c (default), 0 k_z_step, 1 k_z_step_tma (sf_set_z_kernel)
  ZMaps* zmaps = nullptr;        // tensor maps of k_z_step_tma's inputs (null: not supported here)
  int* zerr = nullptr;           // set on the device by a k_z_step_tma wait that ran out
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [linear][parity]
  long long launches = 0;
  long long launches_per_step[2] = {0, 0};
  // sf_step_host_async: copy streams, two staging buffers per direction and
  // the events that order them with the solver's stream
  struct HostPipe {
    cudaStream_t h2d = nullptr, d2h = nullptr;
    float2* in[2] = {nullptr, nullptr};
    float2* out[2] = {nullptr, nullptr};
    cudaEvent_t ev_in[2] = {nullptr, nullptr};       // input copied to in[b]
    cudaEvent_t ev_used[2] = {nullptr, nullptr};     // in[b] taken into the state
    cudaEvent_t ev_done[2] = {nullptr, nullptr};     // result in out[b]
    cudaEvent_t ev_drained[2] = {nullptr, nullptr};  // out[b] copied to the host
    long long k = 0;
  };
  HostPipe* pipe = nullptr;
};

static const double kBeta[3] = {1.0, 25.0 / 8.0, 9.0 / 4.0};     // IMEXRK.h:631
static const double kZeta[3] = {0.0, -17.0 / 8.0, -5.0 / 4.0};   // IMEXRK.h:632

static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
static int ilog2(int n) { int l = 0; while ((1 << l) < n) l++; return l; }

// k(n) of Differentiation.cpp:113-132
static std::vector<double> kint(int n) {
  std::vector<double> k(n, 0.0);
  if (n == 1) return k;
  int idx = 0;
  for (int v = 0; v <= n / 3; v++) k[idx++] = v;
  for (int v = 0; v < n - 2 * (n / 3) - 1; v++) k[idx++] = 0;
  for (int v = -n / 3; v <= -1; v++) k[idx++] = v;
  return k;
}

static void free_all(sf_solver* s) {
  for (int l = 0; l < 2; l++)
    for (int p = 0; p < 2; p++)
      if (s->graph[l][p]) cudaGraphExecDestroy(s->graph[l][p]);
  delete s->zmaps;
  s->zmaps = nullptr;
  void* ptrs[] = {s->zerr, s->amix, s->adir, s->S[0], s->S[1], s->rold, s->rnl, s->qbuf, s->mixin, s->mixout, s->base, s->zc, s->fa,
                  s->fc, s->inv_den, s->kx, s->ky, s->Ri, s->Ubar, s->dBdz, s->bands, s->kxd, s->kyd,
                  s->red, s->tw, s->stage_ref};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (sf_solver::HostPipe* P = s->pipe) {
    if (P->h2d) cudaStreamSynchronize(P->h2d);
    if (P->d2h) cudaStreamSynchronize(P->d2h);
    for (int b = 0; b < 2; b++) {
      if (P->in[b]) cudaFree(P->in[b]);
      if (P->out[b]) cudaFree(P->out[b]);
      cudaEvent_t* evs[] = {&P->ev_in[b], &P->ev_used[b], &P->ev_done[b], &P->ev_drained[b]};
      for (cudaEvent_t* e : evs)
        if (*e) cudaEventDestroy(*e);
    }
    if (P->h2d) cudaStreamDestroy(P->h2d);
    if (P->d2h) cudaStreamDestroy(P->d2h);
    delete P;
    s->pipe = nullptr;
  }
  if (s->xy.y1) cudaStreamDestroy(s->xy.y1);
  if (s->xy.y2) cudaStreamDestroy(s->xy.y2);
  {
    cudaEvent_t* evs[] = {&s->xy.fork, &s->xy.join};
    for (cudaEvent_t* e : evs)
      if (*e) cudaEventDestroy(*e);
    for (int b = 0; b < kMaxBands; b++) {
      if (s->xy.ev_ify[b]) cudaEventDestroy(s->xy.ev_ify[b]);
      if (s->xy.ev_x[b]) cudaEventDestroy(s->xy.ev_x[b]);
    }
  }
  if (s->st) cudaStreamDestroy(s->st);
}

static void drop_graphs(sf_solver* s) {
  for (int l = 0; l < 2; l++)
    for (int p = 0; p < 2; p++)
      if (s->graph[l][p]) {
        cudaGraphExecDestroy(s->graph[l][p]);
        s->graph[l][p] = nullptr;
      }
}

// Tridiagonal rows of every factor set, per row only (a_j, c_j), following
// UpdateForTimestep (IMEXRK.h:502-545) and the Laplacian (IMEXRK.h:55-78).
static void build_rows(const sf_solver* s, const std::vector<double>& b6, std::vector<float>& fa,
                       std::vector<float>& fc) {
  const int N = s->g.N3;
  fa.assign((size_t)kNumFS * N, 0.f);
  fc.assign((size_t)kNumFS * N, 0.f);
  for (int fs = 0; fs < kNumFS; fs++) {
    const bool lap = fs == kFS_Lap;
    const int fam = lap ? 0 : fs / 3, k = lap ? 0 : fs % 3;
    const bool dir = fam == 2;
    const double sh = 0.5 * (double)s->h[k];
    const double dre = fam == 1 ? s->Re * s->Pr : s->Re;
    const double* lo = &b6[(dir ? 3 : 0) * N];
    const double* up = &b6[(dir ? 5 : 2) * N];
    for (int j = 0; j < N; j++) {
      double a = lap ? lo[j] : -(sh * lo[j]) / dre;
      double c = lap ? up[j] : -(sh * up[j]) / dre;
      if (!dir) {
        if (j == 0) c = 0;
        if (j == 1) { a = 0; c = -1; }
        if (j == N - 2) { a = 1; c = 0; }
        if (j == N - 1) { a = 0; c = 0; }
      } else {
        if (j <= 2 || j >= N - 2) { a = 0; c = 0; }
      }
      if (j == 0) a = 0;
      fa[(size_t)fs * N + j] = (float)a;
      fc[(size_t)fs * N + j] = (float)c;
    }
  }
}

static int refactor(sf_solver* s) {
  // IMEXRK.h:506-508: h = deltaT * {8,2,5}/15, stored in stratifloat
  s->h[0] = (float)(s->dt * 8.0 / 15.0);
  s->h[1] = (float)(s->dt * 2.0 / 15.0);
  s->h[2] = (float)(s->dt * 5.0 / 15.0);
  const int N = s->g.N3;
  std::vector<double> b6(6 * (size_t)N);
  CK(cudaMemcpy(b6.data(), s->bands, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost));
  std::vector<float> fa, fc;
  build_rows(s, b6, fa, fc);
  CK(cudaMemcpyAsync(s->fa, fa.data(), sizeof(float) * fa.size(), cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->fc, fc.data(), sizeof(float) * fc.size(), cudaMemcpyHostToDevice, s->st));
  s->launches += launch_factor(s->g, s->bands, s->kxd, s->kyd, s->h[0], s->h[1], s->h[2], s->Re, s->Pr,
                               s->inv_den, s->st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->st));
  drop_graphs(s);
  return SF_OK;
}

static StageArgs stage_args(sf_solver* s, int k, int cur, bool linear) {
  StageArgs a{};
  a.g = s->g;
  a.S = s->S[cur];
  a.Sn = s->S[1 - cur];
  a.rold = s->rold;
  a.rnl = s->rnl;
  a.qbuf = s->qbuf;
  a.mixin = s->mixin;
  a.mixout = s->mixout;
  a.zc = s->zc;
  a.fa = s->fa;
  a.fc = s->fc;
  a.inv_den = s->inv_den;
  a.kx = s->kx;
  a.ky = s->ky;
  a.Ri = s->Ri;
  a.Ubar = s->Ubar;
  a.dBdz = s->dBdz;
  a.tw = s->tw;
  a.base = s->base;
  a.stage = k;
  a.linear = linear ? 1 : 0;
  a.tlm = linear ? 0 : s->tlm;
  a.run_offset = 0;
  a.xslabs = s->xslabs;
  a.zchunks = s->zchunks;
  a.xgroups = s->xgroups;
  a.xkernel = s->xkernel;
  a.zkernel = s->zkernel;
  a.zmaps = s->zmaps;
  a.zerr = s->zerr;
  const float h = s->h[k];
  a.h = h;
  a.hz = h * (float)kZeta[k];   // (h[k]*zeta[k]) in stratifloat
  a.hb = h * (float)kBeta[k];
  a.cv = 0.5f * h / (float)s->Re;
  a.cb = 0.5f * h / (float)s->Re / (float)s->Pr;
  a.pm = 1.0f / h;             // RemoveDivergence(1/h[k])
  return a;
}

// one IMEXRK::TimeStep (IMEXRK.cpp:8-24) starting from state buffer `par`
static int record_step(sf_solver* s, int par, bool linear) {
  int n = 0;
  int cur = par;
  for (int k = 0; k < 3; k++) {
    StageArgs a = stage_args(s, k, cur, linear);
    s->xy.bands = s->xy_bands;
    n += launch_stage(a, s->st, nullptr, s->g.dim3 && s->xy.y1 ? &s->xy : nullptr);
    cur = 1 - cur;
  }
  return n;
}

static int ensure_graph(sf_solver* s, bool linear, int par) {
  if (s->graph[linear][par]) return SF_OK;
  cudaGraph_t gr;
  CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
  int n = record_step(s, par, linear);
  cudaError_t e = cudaStreamEndCapture(s->st, &gr);
  if (e != cudaSuccess) return fail(SF_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&s->graph[linear][par], gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) return fail(SF_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  s->launches_per_step[linear] = n;
  return SF_OK;
}

// accessors for the other translation units (vector store)
const Geo& sf_solver_geo(const sf_solver* s) { return s->g; }
const float* sf_solver_zc(const sf_solver* s) { return s->zc; }
float2* sf_solver_state(sf_solver* s, int run) { return s->S[s->cur] + (size_t)run * 5 * s->g.fblk; }
cudaStream_t sf_solver_stream(const sf_solver* s) { return s->st; }
const std::vector<double>& sf_solver_z(const sf_solver* s, int which) { return which == 0 ? s->zN : s->zfN; }
const float2* sf_solver_tw(const sf_solver* s) { return s->tw; }
const float* sf_solver_ubar(const sf_solver* s, int run) { return s->Ubar + (size_t)run * s->g.N3; }
void sf_solver_count_launches(sf_solver* s, int n) { s->launches += n; }

extern "C" {

const char* sf_last_error(void) { return g_err.c_str(); }

int sf_create(const sf_grid* grid, const sf_flow* flow, double dt, int device, sf_solver** out) {
  if (!grid || !flow || !out) return fail(SF_EINVAL, "null argument");
  const int N1 = grid->N1, N2 = grid->N2, N3 = grid->N3, nrun = grid->nrun;
  if (!pow2(N1) || N1 < 16 || N1 > kMaxN) return fail(SF_EINVAL, "N1 must be a power of two in [16,512]");
  if (!(N2 == 1 || (pow2(N2) && N2 >= 16 && N2 <= 256)))
    return fail(SF_EINVAL, "N2 must be 1 or a power of two in [16,256]");
  if (N3 % 4 != 0 || N3 < 16 || N3 > 1024) return fail(SF_EINVAL, "N3 must be a multiple of 4 in [16,1024]");
  if (nrun < 1) return fail(SF_EINVAL, "nrun must be >= 1");
  if (!(dt > 0) || !(flow->Re > 0) || !(flow->Pr > 0) || !(flow->L1 > 0) || !(flow->L3 > 0) ||
      (N2 > 1 && !(flow->L2 > 0)))
    return fail(SF_EINVAL, "dt, Re, Pr, L1, L3 (and L2 in 3D) must be positive");
  CK(cudaSetDevice(device));
  sf_solver* s = new sf_solver();
  s->device = device;
  s->L1 = flow->L1; s->L2 = flow->L2; s->L3 = flow->L3; s->Re = flow->Re; s->Pr = flow->Pr; s->dt = dt;
  Geo& g = s->g;
  g.N1 = N1; g.N2 = N2; g.N3 = N3; g.nrun = nrun;
  g.dim3 = N2 > 1 ? 1 : 0;
  g.K1 = N1 / 3;
  g.Ky = g.dim3 ? N2 / 3 : 1;
  g.K2 = g.dim3 ? 2 * (N2 / 3) - 1 : 1;
  g.P = g.K1 * g.K2;
  g.Pp = (g.P + 15) / 16 * 16;
  g.logN1 = ilog2(N1);
  g.logN2 = ilog2(N2);
  g.inv_n12 = 1.0f / (float)(N1 * N2);
  g.fblk = (long long)N3 * g.Pp;
  g.mblk = (long long)N3 * N2 * g.K1;

  auto cleanup_fail = [&](int code) { free_all(s); delete s; return code; };
#define CKC(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e__ = (call);                                                                      \
    if (e__ != cudaSuccess) {                                                                      \
      fail(e__ == cudaErrorMemoryAllocation ? SF_ENOMEM : SF_ECUDA,                                \
           std::string(#call) + ": " + cudaGetErrorString(e__));                                   \
      return cleanup_fail(e__ == cudaErrorMemoryAllocation ? SF_ENOMEM : SF_ECUDA);                \
    }                                                                                              \
  } while (0)

  if (prepare_kernels() != 0 || prepare_adjoint_kernels() != 0)
    return cleanup_fail(fail(SF_ECUDA, "cudaFuncSetAttribute failed"));
  CKC(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  if (g.dim3) {
    CKC(cudaStreamCreateWithFlags(&s->xy.y1, cudaStreamNonBlocking));
    CKC(cudaStreamCreateWithFlags(&s->xy.y2, cudaStreamNonBlocking));
    CKC(cudaEventCreateWithFlags(&s->xy.fork, cudaEventDisableTiming));
    CKC(cudaEventCreateWithFlags(&s->xy.join, cudaEventDisableTiming));
    for (int b = 0; b < kMaxBands; b++) {
      CKC(cudaEventCreateWithFlags(&s->xy.ev_ify[b], cudaEventDisableTiming));
      CKC(cudaEventCreateWithFlags(&s->xy.ev_x[b], cudaEventDisableTiming));
    }
  }
  const size_t cb = sizeof(float2);
  CKC(cudaMalloc(&s->S[0], cb * nrun * 5 * g.fblk));
  CKC(cudaMalloc(&s->S[1], cb * nrun * 5 * g.fblk));
  CKC(cudaMalloc(&s->rold, cb * nrun * 4 * g.fblk));
  CKC(cudaMalloc(&s->rnl, cb * nrun * 4 * g.fblk));
  CKC(cudaMalloc(&s->qbuf, cb * nrun * g.fblk));
  CKC(cudaMemset(s->S[0], 0, cb * nrun * 5 * g.fblk));
  CKC(cudaMemset(s->S[1], 0, cb * nrun * 5 * g.fblk));
  CKC(cudaMemset(s->rold, 0, cb * nrun * 4 * g.fblk));
  CKC(cudaMemset(s->rnl, 0, cb * nrun * 4 * g.fblk));
  CKC(cudaMemset(s->qbuf, 0, cb * nrun * g.fblk));
  if (g.dim3) {
    CKC(cudaMalloc(&s->mixin, cb * nrun * 4 * g.mblk));
    CKC(cudaMalloc(&s->mixout, cb * nrun * 8 * g.mblk));
  }
  CKC(cudaMalloc(&s->zc, sizeof(float) * ZC_COUNT * N3));
  CKC(cudaMalloc(&s->fa, sizeof(float) * kNumFS * N3));
  CKC(cudaMalloc(&s->fc, sizeof(float) * kNumFS * N3));
  CKC(cudaMalloc(&s->inv_den, sizeof(float) * kNumFS * g.fblk));
  CKC(cudaMalloc(&s->kx, sizeof(float) * g.K1));
  CKC(cudaMalloc(&s->ky, sizeof(float) * g.K2));
  CKC(cudaMalloc(&s->kxd, sizeof(double) * g.K1));
  CKC(cudaMalloc(&s->kyd, sizeof(double) * g.K2));
  CKC(cudaMalloc(&s->bands, sizeof(double) * 6 * N3));
  CKC(cudaMalloc(&s->Ri, sizeof(float) * nrun));
  CKC(cudaMalloc(&s->Ubar, sizeof(float) * nrun * N3));
  CKC(cudaMalloc(&s->dBdz, sizeof(float) * nrun * N3));
  CKC(cudaMalloc(&s->red, sizeof(double) * 4 * nrun));
  CKC(cudaMalloc(&s->tw, sizeof(float2) * kMaxN));
  CKC(cudaMalloc(&s->stage_ref, sizeof(float2) * (size_t)(N1 / 2 + 1) * N2 * N3));

  // ---- vertical grid, Field.cpp:3-83, in FP64 ----
  const int N = N3;
  std::vector<double> z(N, 0.0), zf(N, 0.0), DY(N, 0.0), DYF(N, 0.0);
  {
    const double cs = 2.0, L = flow->L3;
    const double step = 2.0 / (double)(N - 2);   // Eigen LinSpaced(N-1,-1,1)
    for (int i = 0; i < N - 1; i++) {
      double x = (i == N - 2) ? 1.0 : -1.0 + i * step;
      z[i + 1] = L * (cs * std::pow(x, 7) + x) / (cs + 1);
    }
    double off = (z[1] + z[2]) / 2;
    for (int i = 1; i < N; i++) z[i] *= -L / off;
    for (int i = 1; i <= N - 2; i++) zf[i] = 0.5 * (z[i] + z[i + 1]);
    zf[0] = 2 * zf[1] - zf[2];
    zf[N - 1] = 2 * zf[N - 2] - zf[N - 3];
    for (int i = 1; i < N; i++) DY[i] = zf[i] - zf[i - 1];
    for (int i = 1; i <= N - 2; i++) DYF[i] = z[i + 1] - z[i];
    DYF[N - 1] = DYF[N - 2];
    DYF[0] = DYF[1];
  }
  s->zN = z;
  s->zfN = zf;
  // ---- bands, Differentiation.cpp:6-110 ----
  std::vector<double> b6(6 * (size_t)N, 0.0);   // d2n lo,di,up ; d2d lo,di,up
  std::vector<float> zc((size_t)ZC_COUNT * N, 0.f);
  for (int j = 1; j < N - 1; j++) {
    b6[0 * N + j] = 1 / DY[j] / DYF[j];
    b6[1 * N + j] = -1 / DY[j] / DYF[j] - 1 / DY[j + 1] / DYF[j];
    b6[2 * N + j] = 1 / DY[j + 1] / DYF[j];
  }
  for (int j = 2; j < N - 1; j++) {
    b6[3 * N + j] = 1 / DYF[j - 1] / DY[j];
    b6[4 * N + j] = -1 / DYF[j - 1] / DY[j] - 1 / DYF[j] / DY[j];
    b6[5 * N + j] = 1 / DYF[j] / DY[j];
  }
  for (int b = 0; b < 6; b++)
    for (int j = 0; j < N; j++) zc[(size_t)(ZC_D2N_LO + b) * N + j] = (float)b6[(size_t)b * N + j];
  for (int j = 2; j <= N - 1; j++) {
    zc[(size_t)ZC_DND_LO * N + j] = (float)(-1 / DY[j]);
    zc[(size_t)ZC_DND_DI * N + j] = (float)(1 / DY[j]);
  }
  for (int j = 1; j <= N - 1; j++) {
    zc[(size_t)ZC_DDN_DI * N + j] = (float)(-1 / DYF[j]);
    if (j < N - 1) zc[(size_t)ZC_DDN_UP * N + j] = (float)(1 / DYF[j]);
    zc[(size_t)ZC_FULL_LO * N + j] = (float)(DYF[j] / (2 * DY[j]));
    zc[(size_t)ZC_FULL_DI * N + j] = (float)(DYF[j - 1] / (2 * DY[j]));
    zc[(size_t)ZC_TILDE_LO * N + j] = (float)(DYF[j - 1] / (2 * DY[j]));
    zc[(size_t)ZC_TILDE_DI * N + j] = (float)(DYF[j] / (2 * DY[j]));
  }
  for (int k = 1; k < N - 1; k++) zc[(size_t)ZC_WZN * N + k] = (float)(z[k + 1] - z[k]);
  for (int k = 2; k < N - 1; k++) zc[(size_t)ZC_WZD * N + k] = (float)(zf[k] - zf[k - 1]);
  CKC(cudaMemcpy(s->bands, b6.data(), sizeof(double) * 6 * N, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(s->zc, zc.data(), sizeof(float) * zc.size(), cudaMemcpyHostToDevice));
  // ---- Fourier wavenumbers, Differentiation.cpp:113-160 ----
  {
    const double pi = 3.141592653589793238462;
    auto k1 = kint(N1), k2 = kint(N2);
    std::vector<double> kxd(g.K1), kyd(g.K2);
    std::vector<float> kxf(g.K1), kyf(g.K2);
    for (int j = 0; j < g.K1; j++) kxd[j] = k1[j] * (2 * pi) / flow->L1;
    for (int q = 0; q < g.K2; q++) {
      if (!g.dim3) { kyd[q] = 0; continue; }
      int n2 = q < g.Ky ? q : q + N2 - g.K2;
      kyd[q] = k2[n2] * (2 * pi) / flow->L2;
    }
    for (int j = 0; j < g.K1; j++) kxf[j] = (float)kxd[j];
    for (int q = 0; q < g.K2; q++) kyf[q] = (float)kyd[q];
    CKC(cudaMemcpy(s->kxd, kxd.data(), sizeof(double) * g.K1, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->kyd, kyd.data(), sizeof(double) * g.K2, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->kx, kxf.data(), sizeof(float) * g.K1, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->ky, kyf.data(), sizeof(float) * g.K2, cudaMemcpyHostToDevice));
  }
  // ---- twiddles e^{-2 pi i k/kMaxN}, FP64 -> FP32 ----
  {
    std::vector<float2> tw(kMaxN);
    for (int k = 0; k < kMaxN; k++) {
      double a = -2.0 * 3.141592653589793238462 * k / kMaxN;
      tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    CKC(cudaMemcpy(s->tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice));
  }
  s->hRi.assign(nrun, 0.f);
  CKC(cudaMemset(s->Ri, 0, sizeof(float) * nrun));
  CKC(cudaMemset(s->Ubar, 0, sizeof(float) * nrun * N3));
  {
    std::vector<float> ones((size_t)nrun * N3, 1.f);
    CKC(cudaMemcpy(s->dBdz, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice));
  }
  CKC(cudaMalloc(&s->zerr, sizeof(int)));
  CKC(cudaMemset(s->zerr, 0, sizeof(int)));
  if (zstep_tma_supported(g)) {
    s->zmaps = new ZMaps();
    if (zstep_tma_maps(g, s->S[0], s->S[1], s->rnl, s->rold, s->inv_den, s->zmaps) != 0) {
      delete s->zmaps;   // no tensor maps: k_z_step serves every launch
      s->zmaps = nullptr;
    }
  }
  int rc = refactor(s);
  if (rc != SF_OK) return cleanup_fail(rc);
#undef CKC
  *out = s;
  return SF_OK;
}

int sf_destroy(sf_solver* s) {
  if (!s) return SF_OK;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->st);
  free_all(s);
  delete s;
  return SF_OK;
}

int sf_set_dt(sf_solver* s, double dt) {
  if (!s || !(dt > 0)) return fail(SF_EINVAL, "dt must be positive");
  s->dt = dt;
  return refactor(s);
}

int sf_set_ri(sf_solver* s, int run, double Ri) {
  if (!s || run < 0 || run >= s->g.nrun) return fail(SF_EINVAL, "bad run");
  s->hRi[run] = (float)Ri;
  CK(cudaMemcpyAsync(s->Ri + run, &s->hRi[run], sizeof(float), cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return SF_OK;
}

int sf_set_background(sf_solver* s, int run, const double* U, const double* dBdz) {
  if (!s || run < 0 || run >= s->g.nrun || !U || !dBdz) return fail(SF_EINVAL, "bad argument");
  const int N = s->g.N3;
  std::vector<float> u(N), d(N);
  for (int j = 0; j < N; j++) { u[j] = (float)U[j]; d[j] = (float)dBdz[j]; }
  CK(cudaMemcpyAsync(s->Ubar + (size_t)run * N, u.data(), sizeof(float) * N, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->dBdz + (size_t)run * N, d.data(), sizeof(float) * N, cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return SF_OK;
}

static size_t ref_elems(const sf_solver* s) { return (size_t)(s->g.N1 / 2 + 1) * s->g.N2 * s->g.N3; }

int sf_set_field(sf_solver* s, int run, int field, const float* ref) {
  if (!s || run < 0 || run >= s->g.nrun || field < 0 || field > 4 || !ref) return fail(SF_EINVAL, "bad argument");
  CK(cudaMemcpyAsync(s->stage_ref, ref, sizeof(float2) * ref_elems(s), cudaMemcpyHostToDevice, s->st));
  float2* dst = s->S[s->cur] + ((size_t)run * 5 + field) * s->g.fblk;
  if (field == SF_U2 && !s->g.dim3) {
    CK(cudaMemsetAsync(dst, 0, sizeof(float2) * s->g.fblk, s->st));   // CopyToSolver zeroes u2 in 2D
  } else {
    s->launches += launch_gather_ref(s->g, s->stage_ref, dst, s->st);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s->st));
  return SF_OK;
}

int sf_get_field(sf_solver* s, int run, int field, float* ref) {
  if (!s || run < 0 || run >= s->g.nrun || field < 0 || field > 4 || !ref) return fail(SF_EINVAL, "bad argument");
  CK(cudaMemsetAsync(s->stage_ref, 0, sizeof(float2) * ref_elems(s), s->st));
  const float2* src = s->S[s->cur] + ((size_t)run * 5 + field) * s->g.fblk;
  s->launches += launch_scatter_ref(s->g, src, s->stage_ref, s->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ref, s->stage_ref, sizeof(float2) * ref_elems(s), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  return SF_OK;
}

int sf_set_state_kept(sf_solver* s, const float* host) {
  if (!s || !host) return fail(SF_EINVAL, "bad argument");
  CK(cudaMemcpyAsync(s->S[s->cur], host, sizeof(float2) * s->g.nrun * 5 * s->g.fblk, cudaMemcpyHostToDevice,
                     s->st));
  CK(cudaStreamSynchronize(s->st));
  return SF_OK;
}

int sf_get_state_kept(sf_solver* s, float* host) {
  if (!s || !host) return fail(SF_EINVAL, "bad argument");
  CK(cudaMemcpyAsync(host, s->S[s->cur], sizeof(float2) * s->g.nrun * 5 * s->g.fblk, cudaMemcpyDeviceToHost,
                     s->st));
  CK(cudaStreamSynchronize(s->st));
  return SF_OK;
}

int sf_state_device(sf_solver* s, void** dptr, size_t* bytes) {
  if (!s || !dptr) return fail(SF_EINVAL, "bad argument");
  *dptr = s->S[s->cur];
  if (bytes) *bytes = sizeof(float2) * s->g.nrun * 5 * s->g.fblk;
  return SF_OK;
}

int sf_set_state_device(sf_solver* s, const void* dptr) {
  if (!s || !dptr) return fail(SF_EINVAL, "bad argument");
  CK(cudaMemcpyAsync(s->S[s->cur], dptr, sizeof(float2) * s->g.nrun * 5 * s->g.fblk, cudaMemcpyDeviceToDevice,
                     s->st));
  return SF_OK;
}

int sf_remove_divergence(sf_solver* s, double pm) {
  if (!s) return fail(SF_EINVAL, "null solver");
  StageArgs a = stage_args(s, 0, s->cur, false);
  a.Sn = s->S[s->cur];   // in place
  a.pm = (float)pm;
  s->launches += launch_project(a, s->st);
  CK(cudaGetLastError());
  return SF_OK;
}

int sf_prepare(sf_solver* s) {
  // FilterAll is implicit (only kept modes are stored); RemoveDivergence(0)
  return sf_remove_divergence(s, 0.0);
}

static int step_impl(sf_solver* s, int nsteps, bool linear) {
  if (!s || nsteps < 0) return fail(SF_EINVAL, "bad argument");
  if (linear && !s->base_set) return fail(SF_ESTATE, "sf_step_linear needs sf_set_base first");
  for (int i = 0; i < nsteps; i++) {
    int rc = ensure_graph(s, linear, s->cur);
    if (rc != SF_OK) return rc;
    CK(cudaGraphLaunch(s->graph[linear][s->cur], s->st));
    s->launches += s->launches_per_step[linear];
    s->cur = 1 - s->cur;
  }
  CK(cudaGetLastError());
  return SF_OK;
}

int sf_step(sf_solver* s, int nsteps) { return step_impl(s, nsteps, false); }

int sf_step_host_async(sf_solver* s, const float* host_in, float* host_out, int nsteps) {
  if (!s || !host_in || !host_out || nsteps < 0) return fail(SF_EINVAL, "bad argument");
  const size_t bytes = sizeof(float2) * s->g.nrun * 5 * s->g.fblk;
  if (!s->pipe) {
    s->pipe = new sf_solver::HostPipe();
    sf_solver::HostPipe& P = *s->pipe;
    CK(cudaStreamCreateWithFlags(&P.h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&P.d2h, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++) {
      CK(cudaMalloc(&P.in[b], bytes));
      CK(cudaMalloc(&P.out[b], bytes));
      cudaEvent_t* evs[] = {&P.ev_in[b], &P.ev_used[b], &P.ev_done[b], &P.ev_drained[b]};
      for (cudaEvent_t* e : evs) CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
  }
  sf_solver::HostPipe& P = *s->pipe;
  const int b = (int)(P.k & 1);
  // the input, once the call two back has taken staging buffer b into its state
  CK(cudaStreamWaitEvent(P.h2d, P.ev_used[b], 0));
  CK(cudaMemcpyAsync(P.in[b], host_in, bytes, cudaMemcpyHostToDevice, P.h2d));
  CK(cudaEventRecord(P.ev_in[b], P.h2d));
  CK(cudaStreamWaitEvent(s->st, P.ev_in[b], 0));
  CK(cudaMemcpyAsync(s->S[s->cur], P.in[b], bytes, cudaMemcpyDeviceToDevice, s->st));
  CK(cudaEventRecord(P.ev_used[b], s->st));
  int rc = step_impl(s, nsteps, false);
  if (rc != SF_OK) return rc;
  // the result, once the output copy of the call two back has left buffer b
  CK(cudaStreamWaitEvent(s->st, P.ev_drained[b], 0));
  CK(cudaMemcpyAsync(P.out[b], s->S[s->cur], bytes, cudaMemcpyDeviceToDevice, s->st));
  CK(cudaEventRecord(P.ev_done[b], s->st));
  CK(cudaStreamWaitEvent(P.d2h, P.ev_done[b], 0));
  CK(cudaMemcpyAsync(host_out, P.out[b], bytes, cudaMemcpyDeviceToHost, P.d2h));
  CK(cudaEventRecord(P.ev_drained[b], P.d2h));
  P.k++;
  return SF_OK;
}
int sf_step_linear(sf_solver* s, int nsteps) { return step_impl(s, nsteps, true); }

int sf_set_base(sf_solver* s, int run, const float* u1, const float* u2, const float* u3, const float* b) {
  if (!s || run < 0 || run >= s->g.nrun || !u1 || !u3 || !b) return fail(SF_EINVAL, "bad argument");
  const Geo& g = s->g;
  if (!s->base) {
    CK(cudaMalloc(&s->base, sizeof(float) * (size_t)g.nrun * 4 * g.N3 * g.N2 * g.N1));
    CK(cudaMemset(s->base, 0, sizeof(float) * (size_t)g.nrun * 4 * g.N3 * g.N2 * g.N1));
    drop_graphs(s);   // graphs captured before hold a null base pointer
  }
  float* scratch = nullptr;
  if (g.dim3) CK(cudaMalloc(&scratch, sizeof(float2) * g.mblk));
  const float* src[4] = {u1, u2, u3, b};
  for (int f = 0; f < 4; f++) {
    float* dst = s->base + ((size_t)run * 4 + f) * g.N3 * g.N2 * g.N1;
    if (f == 1 && (!g.dim3 || !u2)) {
      CK(cudaMemsetAsync(dst, 0, sizeof(float) * (size_t)g.N3 * g.N2 * g.N1, s->st));
      continue;
    }
    CK(cudaMemcpyAsync(s->stage_ref, src[f], sizeof(float2) * ref_elems(s), cudaMemcpyHostToDevice, s->st));
    s->launches += launch_gather_ref(g, s->stage_ref, s->qbuf, s->st);
    s->launches += launch_base_nodal(g, s->qbuf, f, dst, s->tw, scratch, s->st);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s->st));
  if (scratch) cudaFree(scratch);
  s->base_set = true;
  return SF_OK;
}

int sf_set_base_device(sf_solver* s, int run, const void* kept_state) {
  if (!s || run < 0 || run >= s->g.nrun || !kept_state) return fail(SF_EINVAL, "bad argument");
  const Geo& g = s->g;
  if (!s->base) {
    CK(cudaMalloc(&s->base, sizeof(float) * (size_t)g.nrun * 4 * g.N3 * g.N2 * g.N1));
    CK(cudaMemset(s->base, 0, sizeof(float) * (size_t)g.nrun * 4 * g.N3 * g.N2 * g.N1));
    drop_graphs(s);   // graphs captured before hold a null base pointer
  }
  float* scratch = nullptr;
  if (g.dim3) CK(cudaMalloc(&scratch, sizeof(float2) * g.mblk));
  const float2* src = static_cast<const float2*>(kept_state);
  for (int f = 0; f < 4; f++) {
    float* dst = s->base + ((size_t)run * 4 + f) * g.N3 * g.N2 * g.N1;
    if (f == 1 && !g.dim3) {
      CK(cudaMemsetAsync(dst, 0, sizeof(float) * (size_t)g.N3 * g.N2 * g.N1, s->st));
      continue;
    }
    // through the same staging buffer as sf_set_base (the 3D transform reads
    // a whole state's worth of rows from its input)
    CK(cudaMemcpyAsync(s->qbuf, src + (size_t)f * g.fblk, sizeof(float2) * g.fblk, cudaMemcpyDeviceToDevice, s->st));
    s->launches += launch_base_nodal(g, s->qbuf, f, dst, s->tw, scratch, s->st);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s->st));
  if (scratch) cudaFree(scratch);
  s->base_set = true;
  return SF_OK;
}

int sf_energy(sf_solver* s, int run, double* ke, double* pe) {
  if (!s || run < 0 || run >= s->g.nrun) return fail(SF_EINVAL, "bad argument");
  const Geo& g = s->g;
  CK(cudaMemsetAsync(s->red, 0, sizeof(double) * 4, s->st));
  const float2* st = s->S[s->cur] + (size_t)run * 5 * g.fblk;
  s->launches += launch_energy(g, st, st, 1, s->zc, s->Ri, s->red, s->st);
  CK(cudaGetLastError());
  double h[4];
  CK(cudaMemcpyAsync(h, s->red, sizeof(h), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  // IMEXRK::KE / PE (IMEXRK.h:395-411)
  double e = 0.5 * (h[0] + h[2]);
  if (g.dim3) e += 0.5 * h[1];
  if (ke) *ke = e;
  if (pe) *pe = (double)s->hRi[run] * 0.5 * h[3];
  return SF_OK;
}

int sf_dissipation(sf_solver* s, int run, double* eps, double* chi) {
  if (!s || run < 0 || run >= s->g.nrun) return fail(SF_EINVAL, "bad argument");
  const Geo& g = s->g;
  CK(cudaMemsetAsync(s->red, 0, sizeof(double) * 4, s->st));
  const float2* st = s->S[s->cur] + (size_t)run * 5 * g.fblk;
  s->launches += launch_grad_sq(g, st, 1, s->zc, s->kxd, s->kyd, s->red, s->st);
  CK(cudaGetLastError());
  double h[4];
  CK(cudaMemcpyAsync(h, s->red, sizeof(h), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  double gu = h[0] + h[2];
  if (g.dim3) gu += h[1];
  if (eps) *eps = gu / s->Re;
  if (chi) *chi = (double)s->hRi[run] / (s->Re * s->Pr) * h[3];
  return SF_OK;
}

int sf_dot(sf_solver* sa, int ra, sf_solver* sb, int rb, double* out) {
  if (!sa || !sb || !out || ra < 0 || ra >= sa->g.nrun || rb < 0 || rb >= sb->g.nrun)
    return fail(SF_EINVAL, "bad argument");
  if (sa->g.N1 != sb->g.N1 || sa->g.N2 != sb->g.N2 || sa->g.N3 != sb->g.N3)
    return fail(SF_EINVAL, "grids differ");
  if (sb != sa) CK(cudaStreamSynchronize(sb->st));
  const Geo& g = sa->g;
  CK(cudaMemsetAsync(sa->red, 0, sizeof(double) * 4, sa->st));
  const float2* A = sa->S[sa->cur] + (size_t)ra * 5 * g.fblk;
  const float2* B = sb->S[sb->cur] + (size_t)rb * 5 * g.fblk;
  sa->launches += launch_energy(g, A, B, 1, sa->zc, sa->Ri, sa->red, sa->st);
  CK(cudaGetLastError());
  double h[4];
  CK(cudaMemcpyAsync(h, sa->red, sizeof(h), cudaMemcpyDeviceToHost, sa->st));
  CK(cudaStreamSynchronize(sa->st));
  // StateVector::Dot (StateVector.h:122-134)
  double d = h[0] + h[2] + (double)sa->hRi[ra] * h[3];
  if (g.dim3) d += h[1];
  *out = d;
  return SF_OK;
}

int sf_profile_step(sf_solver* s, int nsteps, int linear, int cap, double* ms, int* nslots) {
  if (!s || nsteps < 1 || !ms || !nslots) return fail(SF_EINVAL, "bad argument");
  if (linear && !s->base_set) return fail(SF_ESTATE, "linear profile needs sf_set_base first");
  const int per = stage_kernel_count(s->g), n = 3 * per;
  if (cap < n) return fail(SF_EINVAL, "ms buffer too small");
  std::vector<cudaEvent_t> ev(n + 1);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(n, 0.0);
  for (int it = 0; it < nsteps; it++) {
    CK(cudaEventRecord(ev[0], s->st));
    for (int k = 0; k < 3; k++) {
      StageArgs a = stage_args(s, k, s->cur, linear != 0);
      s->launches += launch_stage(a, s->st, &ev[1 + k * per]);
      s->cur = 1 - s->cur;
    }
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev[n]));
    for (int i = 0; i < n; i++) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
      acc[i] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int i = 0; i < n; i++) ms[i] = acc[i] / nsteps;
  *nslots = n;
  return SF_OK;
}

int sf_profile_names(sf_solver* s, char* buf, size_t len) {
  if (!s || !buf || len == 0) return fail(SF_EINVAL, "bad argument");
  std::string out;
  // the nonlinear 3D x pass runs as k_xmarch where the solver takes it
  const bool march = s->xkernel == 1 && !s->tlm && xmarch_supported(stage_args(s, 0, s->cur, false));
  // and the z pass as k_z_step_tma
  const StageArgs a0 = stage_args(s, 0, s->cur, false);
  const char* zname = z_step_takes_c(a0) ? "k_z_step_c" : (z_step_takes_tma(a0) ? "k_z_step_tma" : "k_z_step");
  for (int k = 0; k < 3; k++)
    for (int i = 0; i < stage_kernel_count(s->g); i++) {
      if (!out.empty()) out += ",";
      const std::string nm = stage_kernel_name(s->g, i);
      out += (march && nm == "k_xpass") ? std::string("k_xmarch") : nm == "k_z_step" ? std::string(zname) : nm;
    }
  if (out.size() + 1 > len) return fail(SF_EINVAL, "buffer too small");
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return SF_OK;
}

extern "C" int sf_velocity_maxima(sf_solver* s, int run, double* out3);

// IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126); below/above: nrun device states
// in the kept layout [nrun][5][N3][plane] (u1, u2, u3, b used)
int sf_step_adjoint(sf_solver* s, const void* below, const void* above) {
  if (!s || !below || !above) return fail(SF_EINVAL, "bad argument");
  const Geo& g = s->g;
  if (!s->adir) CK(cudaMalloc(&s->adir, sizeof(float2) * (size_t)4 * g.fblk * g.nrun));
  if (g.dim3 && !s->amix) CK(cudaMalloc(&s->amix, sizeof(float2) * (size_t)12 * g.mblk * g.nrun));
  float frac = 0.f;
  int cur = s->cur;
  for (int k = 0; k < 3; k++) {
    StageArgs a = stage_args(s, k, cur, false);
    a.tlm = 0;
    a.amix = s->amix;
    a.adj_invK = 0.5f;   // 1/K, K = 2 (IMEXRK.h:487)
    s->launches += launch_stage_adjoint(a, static_cast<const float2*>(below), static_cast<const float2*>(above), frac,
                                        s->adir, s->st);
    CK(cudaGetLastError());
    cur = 1 - cur;
    frac += s->h[k] / (float)s->dt;   // interpFrac += h[k]/deltaT
  }
  s->cur = cur;
  return SF_OK;
}

int sf_get_runs(sf_solver* s, int* nrun) {
  if (!s || !nrun) return fail(SF_EINVAL, "bad argument");
  *nrun = s->g.nrun;
  return SF_OK;
}

int sf_get_dt(sf_solver* s, double* dt) {
  if (!s || !dt) return fail(SF_EINVAL, "bad argument");
  *dt = s->dt;
  return SF_OK;
}

// IMEXRK::CFL (IMEXRK.h:355-366): (max|U1 + U_|/d1 + max|U2|/d2 + max|U3|/d3) dt,
// d1 = L1/N1, d2 = L2/N2, d3 = z(N3/2+1) - z(N3/2), the smallest gap
int sf_cfl(sf_solver* s, int run, double* cfl) {
  if (!s || !cfl) return fail(SF_EINVAL, "bad argument");
  double m[3];
  int rc = sf_velocity_maxima(s, run, m);
  if (rc) return rc;
  const Geo& g = s->g;
  const double d1 = s->L1 / g.N1, d2 = s->L2 / g.N2, d3 = s->zN[g.N3 / 2 + 1] - s->zN[g.N3 / 2];
  *cfl = (m[0] / d1 + (g.dim3 ? m[1] / d2 : 0.0) + m[2] / d3) * s->dt;
  return SF_OK;
}

int sf_set_xpass_groups(sf_solver* s, int groups) {
  if (!s || groups < 0 || groups > 32) return fail(SF_EINVAL, "groups must be in [0, 32]");
  if (groups != s->xgroups) {
    s->xgroups = groups;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_set_xpass_kernel(sf_solver* s, int kind) {
  if (!s || (kind != 0 && kind != 1)) return fail(SF_EINVAL, "kind must be 0 or 1");
  if (kind != s->xkernel) {
    s->xkernel = kind;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_set_z_kernel(sf_solver* s, int kind) {
  if (!s || kind < 0 || kind > 2) return fail(SF_EINVAL, "kind must be 0, 1 or 2");
  if (kind != s->zkernel) {
    s->zkernel = kind;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_set_z_chunks(sf_solver* s, int chunks) {
  if (!s || !(chunks == 0 || chunks == 8 || chunks == 16)) return fail(SF_EINVAL, "chunks must be 0, 8 or 16");
  if (s->g.N3 < 2 * (chunks ? chunks : 8)) return fail(SF_EINVAL, "too few levels for that many chunks");
  if (chunks != s->zchunks) {
    s->zchunks = chunks;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_set_xy_bands(sf_solver* s, int bands) {
  if (!s || bands < 1 || bands > kMaxBands) return fail(SF_EINVAL, "bands must be in [1, 8]");
  if (bands != s->xy_bands) {
    s->xy_bands = bands;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_set_xpass_slabs(sf_solver* s, int slabs) {
  if (!s || slabs < 0) return fail(SF_EINVAL, "bad argument");
  if (slabs != s->xslabs) {
    s->xslabs = slabs;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_set_tangent(sf_solver* s, int nbase) {
  if (!s) return fail(SF_EINVAL, "null solver");
  if (nbase < 0 || (nbase > 0 && (s->g.nrun <= nbase || s->g.nrun % nbase != 0)))
    return fail(SF_EINVAL, "nbase must divide nrun and be smaller than it (0 switches the mode off)");
  if (nbase != s->tlm) {
    s->tlm = nbase;
    drop_graphs(s);
  }
  return SF_OK;
}

int sf_synchronize(sf_solver* s) {
  if (!s) return fail(SF_EINVAL, "null solver");
  CK(cudaStreamSynchronize(s->st));
  if (s->pipe) {
    CK(cudaStreamSynchronize(s->pipe->h2d));
    CK(cudaStreamSynchronize(s->pipe->d2h));
  }
  if (s->zkernel == 1 && s->zmaps) {
    int h = 0;
    CK(cudaMemcpy(&h, s->zerr, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
      CK(cudaMemset(s->zerr, 0, sizeof(int)));
      return fail(SF_ECUDA, "a z-pass block gave up waiting for its input tiles");
    }
  }
  return SF_OK;
}

int sf_stream(sf_solver* s, void** stream) {
  if (!s || !stream) return fail(SF_EINVAL, "bad argument");
  *stream = (void*)s->st;
  return SF_OK;
}

int sf_launch_count(sf_solver* s, long long* count) {
  if (!s || !count) return fail(SF_EINVAL, "bad argument");
  *count = s->launches;
  return SF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- ensembles
// A batch of independent 2D runs on grids of different sizes: one member
// solver per run (its own buffers, factors, Ri and background), stepped
// together with one launch per RK stage over the work items of every member
// (k_ens_stage: every member's x-pass blocks, then its z-step blocks), captured
// as one CUDA graph per step parity.
struct sf_ensemble {
  int device = 0;
  std::vector<sf_solver*> members;
  cudaStream_t st = nullptr;
  StageArgs* d_args = nullptr;   // [parity][stage][member]
  std::vector<StageArgs> h_args;
  EnsItem *d_x = nullptr, *d_z = nullptr;
  int nx = 0, nz = 0;
  size_t xsmem = 0, zsmem = 0;
  int* d_counters = nullptr;   // [3 stages][1 + nrun] work-item counters of the stage launches
  int* d_xneed = nullptr;      // [nrun] x-pass items per member
  int* d_err = nullptr;        // a z-step item whose wait ran out
  int blocks = 0;              // persistent blocks of a stage launch
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long launches = 0;
};

static void ens_free(sf_ensemble* e) {
  for (cudaGraphExec_t& gx : e->graph)
    if (gx) cudaGraphExecDestroy(gx);
  for (void* p : {(void*)e->d_args, (void*)e->d_x, (void*)e->d_z, (void*)e->d_counters, (void*)e->d_xneed,
                  (void*)e->d_err})
    if (p) cudaFree(p);
  if (e->st) cudaStreamDestroy(e->st);
  for (sf_solver* m : e->members)
    if (m) sf_destroy(m);
  delete e;
}

extern "C" {

int sf_ensemble_create(int nrun, const sf_grid* grids, const sf_flow* flows, const double* dt, int device,
                       sf_ensemble** out) {
  if (nrun < 1 || !grids || !flows || !dt || !out) return fail(SF_EINVAL, "bad argument");
  for (int r = 0; r < nrun; r++)
    if (grids[r].N2 != 1) return fail(SF_EINVAL, "ensemble members are 2D grids (N2 = 1)");
  CK(cudaSetDevice(device));
  if (prepare_ensemble_kernels() != 0) return fail(SF_ECUDA, "cudaFuncSetAttribute failed (ensemble kernels)");
  sf_ensemble* e = new sf_ensemble();
  e->device = device;
  for (int r = 0; r < nrun; r++) {
    sf_grid g = grids[r];
    g.nrun = 1;
    sf_solver* m = nullptr;
    const int rc = sf_create(&g, &flows[r], dt[r], device, &m);
    if (rc != SF_OK) {
      ens_free(e);
      return rc;
    }
    e->members.push_back(m);
  }
  // work items, the largest members first; every x-pass block takes one
  // 4-level slab (S = 4, no carried slabs)
  std::vector<int> order(nrun);
  for (int r = 0; r < nrun; r++) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (long long)grids[a].N1 * grids[a].N3 > (long long)grids[b].N1 * grids[b].N3;
  });
  std::vector<EnsItem> xi, zi;
  std::vector<int> xneed(nrun, 0);
  for (int r : order) {
    const Geo& g = e->members[r]->g;
    const int S = 4;
    xneed[r] = (g.N3 + S - 1) / S;
    for (int c = 0; c < (g.N3 + S - 1) / S; c++) xi.push_back(EnsItem{r, c, S, 1});
    for (int q = 0; q < (g.P + 15) / 16; q++) zi.push_back(EnsItem{r, q, 0, 0});
    e->xsmem = std::max(e->xsmem, ensemble_xpass_smem(g.N1, S));
    e->zsmem = std::max(e->zsmem, ensemble_zstep_smem(g.N3));
  }
  e->nx = (int)xi.size();
  e->nz = (int)zi.size();
  cudaError_t ce = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_x, sizeof(EnsItem) * xi.size());
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_z, sizeof(EnsItem) * zi.size());
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_args, sizeof(StageArgs) * 6 * nrun);
  if (ce == cudaSuccess) ce = cudaMemcpy(e->d_x, xi.data(), sizeof(EnsItem) * xi.size(), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(e->d_z, zi.data(), sizeof(EnsItem) * zi.size(), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_counters, sizeof(int) * 3 * (nrun + 1));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_xneed, sizeof(int) * nrun);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_err, sizeof(int));
  if (ce == cudaSuccess) ce = cudaMemcpy(e->d_xneed, xneed.data(), sizeof(int) * nrun, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemset(e->d_err, 0, sizeof(int));
  if (ce != cudaSuccess) {
    ens_free(e);
    return fail(ce == cudaErrorMemoryAllocation ? SF_ENOMEM : SF_ECUDA, std::string("ensemble: ") + cudaGetErrorString(ce));
  }
  e->h_args.resize((size_t)6 * nrun);
  e->blocks = ensemble_stage_blocks(std::max(e->xsmem, e->zsmem));
  *out = e;
  return SF_OK;
}

int sf_ensemble_destroy(sf_ensemble* e) {
  if (!e) return fail(SF_EINVAL, "null ensemble");
  cudaStreamSynchronize(e->st);
  ens_free(e);
  return SF_OK;
}

int sf_ensemble_member(sf_ensemble* e, int r, sf_solver** s) {
  if (!e || !s || r < 0 || r >= (int)e->members.size()) return fail(SF_EINVAL, "bad argument");
  *s = e->members[r];
  return SF_OK;
}

int sf_ensemble_step(sf_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return fail(SF_EINVAL, "bad argument");
  const int R = (int)e->members.size();
  const int par = e->members[0]->cur;
  for (sf_solver* m : e->members) {
    if (m->cur != par) return fail(SF_ESTATE, "ensemble members are at different state parities");
    if (m->tlm) return fail(SF_ESTATE, "ensemble members cannot be tangent-linear batches");
    CK(cudaStreamSynchronize(m->st));   // the members' own work (set_state, prepare, ...) first
  }
  // the stage arguments of every member for both parities (h, factors and
  // pointers may have changed since the last call); the graphs read them
  // from the device table
  for (int p = 0; p < 2; p++)
    for (int k = 0; k < 3; k++) {
      const int cur = (k == 1) ? 1 - p : p;
      for (int r = 0; r < R; r++) {
        StageArgs a = stage_args(e->members[r], k, cur, false);
        a.xslabs = 1;
        e->h_args[((size_t)p * 3 + k) * R + r] = a;
      }
    }
  CK(cudaMemcpyAsync(e->d_args, e->h_args.data(), sizeof(StageArgs) * e->h_args.size(), cudaMemcpyHostToDevice,
                     e->st));
  for (int p = 0; p < 2; p++) {
    if (e->graph[p]) continue;
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(e->d_counters, 0, sizeof(int) * 3 * (R + 1), e->st);
    for (int k = 0; k < 3; k++) {
      const StageArgs* a = e->d_args + ((size_t)p * 3 + k) * R;
      launch_ens_stage(a, e->d_x, e->nx, e->d_z, e->nz, e->d_counters + (size_t)k * (R + 1), e->d_xneed, e->d_err,
                       e->blocks, std::max(e->xsmem, e->zsmem), e->st);
    }
    cudaError_t ce = cudaStreamEndCapture(e->st, &gr);
    if (ce != cudaSuccess) return fail(SF_ECUDA, std::string("ensemble graph capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&e->graph[p], gr, 0);
    cudaGraphDestroy(gr);
    if (ce != cudaSuccess) return fail(SF_ECUDA, std::string("ensemble graph: ") + cudaGetErrorString(ce));
  }
  int cur = par;
  for (int i = 0; i < nsteps; i++) {
    CK(cudaGraphLaunch(e->graph[cur], e->st));
    e->launches += 3;
    cur = 1 - cur;   // three stages flip the state buffer three times
  }
  for (sf_solver* m : e->members) m->cur = cur;
  CK(cudaGetLastError());
  return SF_OK;
}

int sf_ensemble_profile(sf_ensemble* e, int nsteps, double* ms_x, double* ms_z) {
  if (!e || nsteps < 1 || !ms_x || !ms_z) return fail(SF_EINVAL, "bad argument");
  // the graphs and the argument table, as a step sets them up
  int rc = sf_ensemble_step(e, 0);
  if (rc != SF_OK) return rc;
  const int R = (int)e->members.size();
  int cur = e->members[0]->cur;
  cudaEvent_t ev[7];
  for (cudaEvent_t& x : ev) CK(cudaEventCreate(&x));
  double tx = 0, tz = 0;
  for (int i = 0; i < nsteps; i++) {
    CK(cudaEventRecord(ev[0], e->st));
    for (int k = 0; k < 3; k++) {
      const StageArgs* a = e->d_args + ((size_t)cur * 3 + k) * R;
      launch_xpass_ens(a, e->d_x, e->nx, e->xsmem, e->st);
      CK(cudaEventRecord(ev[1 + 2 * k], e->st));
      launch_zstep_ens(a, e->d_z, e->nz, e->zsmem, e->st);
      CK(cudaEventRecord(ev[2 + 2 * k], e->st));
    }
    CK(cudaEventSynchronize(ev[6]));
    for (int k = 0; k < 3; k++) {
      float a = 0, b = 0;
      CK(cudaEventElapsedTime(&a, ev[2 * k], ev[1 + 2 * k]));
      CK(cudaEventElapsedTime(&b, ev[1 + 2 * k], ev[2 + 2 * k]));
      tx += a;
      tz += b;
    }
    e->launches += 6;
    cur = 1 - cur;
  }
  for (sf_solver* m : e->members) m->cur = cur;
  for (cudaEvent_t& x : ev) cudaEventDestroy(x);
  *ms_x = tx / (3.0 * nsteps);
  *ms_z = tz / (3.0 * nsteps);
  return SF_OK;
}

int sf_ensemble_synchronize(sf_ensemble* e) {
  if (!e) return fail(SF_EINVAL, "null ensemble");
  CK(cudaStreamSynchronize(e->st));
  int h = 0;
  CK(cudaMemcpy(&h, e->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    CK(cudaMemset(e->d_err, 0, sizeof(int)));
    return fail(SF_ECUDA, "an ensemble z-step item gave up waiting for its member's x pass");
  }
  return SF_OK;
}

int sf_ensemble_launch_count(sf_ensemble* e, long long* count) {
  if (!e || !count) return fail(SF_EINVAL, "bad argument");
  *count = e->launches;
  return SF_OK;
}

int sf_ensemble_stream(sf_ensemble* e, void** stream) {
  if (!e || !stream) return fail(SF_EINVAL, "bad argument");
  *stream = (void*)e->st;
  return SF_OK;
}

}  // extern "C"
