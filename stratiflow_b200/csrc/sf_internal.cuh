// Internal declarations shared by the kernels and the C-ABI layer.
//
// Device data layout (all complex values are float2):
//   state   S[2]    [nrun][5][N3][Pp]   u1,u2,u3,b,p per run; two copies,
//                                       stage k reads one and writes the other
//   rold            [nrun][4][N3][Pp]   explicit terms r1,r2,r3,rB of the last
//                                       stage (the zeta term of ExplicitRK)
//   rnl             [nrun][4][N3][Pp]   nonlinear terms of this stage
//   qbuf            [nrun][N3][Pp]      forward-sweep scratch of the pressure solve
//   mixin  (3D)     [nrun][4][N3][N2][K1]  fields after the inverse y transform
//   mixout (3D)     [nrun][8][N3][N2][K1]  x-transformed product combinations
//   base            [nrun][4][N3][N2][N1]  frozen nodal base of the linear step
// Pp = roundup(K1*K2, 16) is the plane stride of one level; mode m = q*K1+j1.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sf {

constexpr int kMaxN = 512;        // largest N1 / N2 of the FFTs
constexpr int kNumFS = 10;        // factor sets: 3 families x 3 stages + Laplacian
constexpr int kFS_Lap = 9;

// per-level coefficient arrays in `zc`, each N3 floats
enum ZC {
  ZC_D2N_LO, ZC_D2N_DI, ZC_D2N_UP,
  ZC_D2D_LO, ZC_D2D_DI, ZC_D2D_UP,
  ZC_DND_LO, ZC_DND_DI,       // ddz Neumann -> Dirichlet (rows 2..N-1)
  ZC_DDN_DI, ZC_DDN_UP,       // ddz Dirichlet -> Neumann (rows 1..N-1)
  ZC_FULL_LO, ZC_FULL_DI,     // ReinterpolateFull
  ZC_TILDE_LO, ZC_TILDE_DI,   // ReinterpolateTilde
  ZC_WZN, ZC_WZD,             // vertical quadrature weights (Integration.h:5-35)
  ZC_COUNT
};

struct Geo {
  int N1, N2, N3;
  int K1, K2, Ky;   // kept x modes, kept y modes, non-negative kept y modes
  int P, Pp;        // kept modes per level, padded plane stride
  int logN1, logN2;
  int nrun;
  int dim3;
  float inv_n12;    // 1/(N1*N2), the ToModal scaling (Field.h:759)
  long long fblk;   // complex elements of one field block: N3*Pp
  long long mblk;   // complex elements of one mixed block: N3*N2*K1
};

struct StageArgs {
  Geo g;
  const float2* S;      // current state [nrun][5][N3][Pp]
  float2* Sn;           // next state
  float2* rold;
  float2* rnl;
  float2* qbuf;
  float2* mixin;
  float2* mixout;
  const float* zc;      // ZC_COUNT x N3
  const float* fa;      // kNumFS x N3 sub-diagonals a_j
  const float* fc;      // kNumFS x N3 super-diagonals c_j
  const float* inv_den; // kNumFS x N3 x Pp, 1/(b_j - a_j C_{j-1}) (FP64-factorised)
  const float* kx;      // K1
  const float* ky;      // K2
  const float* Ri;      // nrun
  const float* Ubar;    // nrun x N3
  const float* dBdz;    // nrun x N3
  const float2* tw;     // kMaxN twiddles e^{-2 pi i k/kMaxN}, the full circle
  const float* base;    // nrun x 4 x N3 x N2 x N1 (linear step only)
  int stage;
  int linear;
  int tlm;          // tangent-linear batch: runs < tlm are nonlinear bases, run r >= tlm
                    // is linearised about the current state of run (r - tlm) % tlm
  int run_offset;   // first run of this launch (x pass)
  int xslabs;       // slabs per x-pass block (0: chosen by the launcher)
  int adjoint;      // adjoint step: no linear buoyancy terms in the z solve
  const float2* adir;   // adjoint step: the direct total state of the substep [nrun][4][N3][Pp]
  float2* amix;         // 3D adjoint step: 12 y-transformed fields [nrun][12][N3][N2][K1]
  float adj_invK;       // adjoint step: 1/K of the mixing objective (IMEXRK.h:487)
  float h, hz, hb, cv, cb, pm;
  // level band of one launch of the y transforms (levels lvl0 .. lvl0+nlvl-1;
  // nlvl = 0: all) and level columns of one x-pass launch (xcol0 .. +xcols-1;
  // xcols = 0: all), for the banded 3D x-y pass
  int lvl0, nlvl, xcol0, xcols;
  int zchunks;      // z chunks per block of the z solves (8 or 16; 0: chosen by the launcher)
  int xgroups;      // lane groups per x-pass block (0: chosen by the launcher)
  int xkernel;      // 3D nonlinear x pass: 1 level-marching lane groups (k_xmarch), 0 slab blocks (k_xpass)
  int zkernel;      // z pass: 0 k_z_step, 1 k_z_step_tma (inputs by the tensor-memory accelerator),
                    // 2 k_z_step_c (one lane per complex mode)
  const void* zmaps;   // host ZMaps of the solver (k_z_step_tma), or null
  int* zerr;           // device word set by a k_z_step_tma wait that ran out
};

// the tensor maps of k_z_step_tma's inputs (each the bytes of one
// CUtensorMap), encoded once per solver, and the state buffers they view
struct alignas(64) ZMap {
  unsigned char bytes[128];
};
struct ZMaps {
  ZMap s[2], rnl, rold, iden;
  const void* sbase[2];
  const void* rbase[3];   // rnl, rold, inv_den
};

// side streams and events of the banded 3D x-y pass: the inverse y
// transforms of every band run on y1, the x passes on the stage's stream, the
// forward y transforms on y2, each band waiting only for what it reads
constexpr int kMaxBands = 8;
struct XYAux {
  cudaStream_t y1, y2;
  cudaEvent_t fork, join;
  cudaEvent_t ev_ify[kMaxBands], ev_x[kMaxBands];
  int bands;
};

// one block's work in an ensemble launch: member solver `run`, block
// coordinate x (x-pass level column or z-solve mode group), and for the x
// pass the slab height S and slabs per block
struct EnsItem {
  int run, x, S, iters;
};
constexpr int kEnsThreads = 256;

// launchers (sf_kernels.cu); each returns the number of kernels launched
int prepare_kernels();
// the z pass with TMA-fed first sweeps (sf_zstep.cu)
bool zstep_tma_supported(const Geo& g);
int zstep_tma_maps(const Geo& g, const float2* S0, const float2* S1, const float2* rnl, const float2* rold,
                   const float* inv_den, ZMaps* out);
int launch_z_step_tma(const StageArgs& a, cudaStream_t st);
bool z_step_takes_tma(const StageArgs& a);
// the z pass with one lane per complex mode (sf_zstep2.cu)
bool zstep_c_supported(const Geo& g);
int launch_z_step_c(const StageArgs& a, cudaStream_t st);
int prepare_zstep_c_kernels();
bool z_step_takes_c(const StageArgs& a);
int prepare_zstep_tma_kernels();
// the 3D nonlinear x pass as level-marching lane groups (sf_xmarch.cu): levels
// t_lo .. t_hi - 1 of every run and y row
bool xmarch_supported(const StageArgs& a);
int launch_xmarch(const StageArgs& a, int t_lo, int t_hi, cudaStream_t st);
int prepare_xmarch_kernels();
// one stage; if ev != nullptr, ev[i] is recorded after the i-th kernel
int launch_stage(const StageArgs& a, cudaStream_t st, cudaEvent_t* ev = nullptr, const XYAux* aux = nullptr);
int stage_kernel_count(const Geo& g);
const char* stage_kernel_name(const Geo& g, int i);
int launch_project(const StageArgs& a, cudaStream_t st);  // RemoveDivergence only
int launch_z_solves(const StageArgs& a, cudaStream_t st);   // CN solve + RemoveDivergence
int launch_fft_y_combos(const StageArgs& a, cudaStream_t st);   // 3D: mixout's 8 combinations -> rnl
// TimeStepAdjoint's stage (sf_adjoint.cu): the direct state of the substep
// into a.adir, then the adjoint x pass and the z solves; 2D
int launch_stage_adjoint(StageArgs a, const float2* below, const float2* above, float frac, float2* adir,
                         cudaStream_t st);
size_t adjoint_smem_needed(const Geo& g);
int prepare_adjoint_kernels();
int launch_factor(const Geo& g, const double* bands, const double* kx, const double* ky,
                  double h0, double h1, double h2, double Re, double Pr, float* inv_den,
                  cudaStream_t st);
int launch_gather_ref(const Geo& g, const float2* ref, float2* kept, cudaStream_t st);
int launch_scatter_ref(const Geo& g, const float2* kept, float2* ref, cudaStream_t st);
int launch_energy(const Geo& g, const float2* Sa, const float2* Sb, int nrun_pairs,
                  const float* zc, const float* Ri, double* out, cudaStream_t st);
// ensembles of 2D solvers of different grids (sf_ensemble): every member's
// x pass in one launch and every member's z step in another; args holds one
// StageArgs per member
size_t ensemble_xpass_smem(int N1, int S);
size_t ensemble_zstep_smem(int N3);
int launch_xpass_ens(const StageArgs* args, const EnsItem* items, int nitems, size_t smem, cudaStream_t st);
int launch_zstep_ens(const StageArgs* args, const EnsItem* items, int nitems, size_t smem, cudaStream_t st);
int prepare_ensemble_kernels();
// the whole stage in one launch of `blocks` persistent blocks over work-item
// counters (counters[0] the next item, counters[1 + r] member r's finished
// x-pass items; cleared before each step)
int launch_ens_stage(const StageArgs* args, const EnsItem* xitems, int nx, const EnsItem* zitems, int nz,
                     int* counters, const int* xneed, int* err, int blocks, size_t smem, cudaStream_t st);
int ensemble_stage_blocks(size_t smem);
int launch_grad_sq(const Geo& g, const float2* S, int nruns, const float* zc, const double* kxd, const double* kyd,
                   double* out, cudaStream_t st);
int launch_base_nodal(const Geo& g, const float2* kept_modal, int field, float* base_out,
                      const float2* tw, float* scratch_mixed, cudaStream_t st);

// ------------------------------------------------------- device helpers ----
#ifdef __CUDACC__
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// (i*k) * a
__device__ __forceinline__ float2 cik(float k, float2 a) { return make_float2(-k * a.y, k * a.x); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// In-place radix-2 decimation-in-time FFT of n = 2^logn points held in shared
// memory at a[0..n), executed by one warp. Unnormalised; sign -1 (forward)
// or +1 (inverse). tw holds e^{-2 pi i k/kMaxN}, k < kMaxN (only k < kMaxN/2 used here).
__device__ __forceinline__ void warp_fft(float2* a, int n, int logn, const float2* __restrict__ tw,
                                         bool inverse, int lane) {
  const int shift = 32 - logn;
  for (int i = lane; i < n; i += 32) {
    int r = (int)(__brev((unsigned)i) >> shift);
    if (i < r) {
      float2 t = a[i];
      a[i] = a[r];
      a[r] = t;
    }
  }
  __syncwarp();
  const int half_n = n >> 1;
  for (int s = 1; s <= logn; s++) {
    const int half = 1 << (s - 1);
    const int twstep = kMaxN >> s;   // e^{-2 pi i pos/(2 half)} = tw[pos * kMaxN/(2 half)]
    for (int bt = lane; bt < half_n; bt += 32) {
      int pos = bt & (half - 1);
      int i0 = ((bt >> (s - 1)) << s) + pos;
      int i1 = i0 + half;
      float2 w = tw[pos * twstep];
      if (inverse) w.y = -w.y;
      float2 x0 = a[i0];
      float2 x1 = cmul(a[i1], w);
      a[i0] = cadd(x0, x1);
      a[i1] = csub(x0, x1);
    }
    __syncwarp();
  }
}
#endif

}  // namespace sf
