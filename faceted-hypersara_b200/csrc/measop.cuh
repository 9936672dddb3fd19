// Measurement operator Phi = G A on the device (see measop.cu).
#pragma once

#include <memory>

#include "common.cuh"
#include "minmax.h"

namespace fhs {

// Read-only view of the operator passed to kernels by value.
struct OpView {
  // tap polynomials (kernel parameters: uniform across threads)
  float py[kMaxTaps][2][kPolyDegree + 1];
  float px[kMaxTaps][2][kPolyDegree + 1];
  // the real taps c_j of the phase-factored form (see cplx.cuh)
  float ry[kMaxTaps][kPolyDegree + 1];
  float rx[kMaxTaps][kPolyDegree + 1];
  int Ny, Nx, Ky, Kx, Jy, Jx;
  int nT0, nT1;      // tiles per axis (kTileCells cells each, last may be partial)
  int nsb0, nsb1;    // sub-bins per axis (kBinCells cells each)
  int nkeys;         // nT0*nT1*kSubPerTile^2 sort keys per channel
  const float2* tab_y;  // [Jy][kTableSamples+1]
  const float2* tab_x;  // [Jx][kTableSamples+1]
  const float* sy;      // [Ny] scaling factors
  const float* sx;      // [Nx]
  const float4* geom;   // per sorted visibility: (fy, fx, kpack bits, weight)
  const float2* vph;    // per sorted visibility: exp(i (om_y + om_x) / 2), the tap phase of the visibility
  const int32_t* sb_off;  // [L][nkeys+1] visibility offsets per sub-bin (channel-relative)
  const int64_t* ch_voff; // [L] first visibility of each channel
  const int32_t* ch_M;    // [L]
};

// A slice of one (channel, tile) for the degridding / gridding kernels.
// Dense tiles are split so that no CTA carries more than a fixed number of
// visibilities (the uv coverage is strongly concentrated near the origin).
struct WorkItem {
  int ch, tile;
  int split, nsplit;
  int slot;   // degrid: block-norm partial slot; grid: partial tile slot (-1: write the grid)
  int pad;
};

// Preconditioned (ellipsoid) dual: pointers read by the tile kernels.
struct PrecondView {
  const float* pu = nullptr;    // [Mtot] diagonal preconditioner pU (sorted order)
  const double2* w = nullptr;   // [Mtot] proj - y, the ellipsoid-projection iterate
  const float* mu = nullptr;    // [L][kMaxBlocksPerChannel] FB step: min of pU over the block
};

// A chunk of one channel's visibilities for the ellipsoid FB passes.
struct FbItem {
  int ch, beg, end, pad;
};

// Sub-bin schedule of one gridding item: the non-empty sub-bins that reach
// the tile (index (j + 1) * 9 + (i + 1) for sub-bin row i, column j in
// [-1, 8), -1 = the ring), grouped by phase (parity of i + 1, j + 1) and
// largest first within a phase.
struct GridPlan {
  int count[4];      // sub-bins per phase
  uint8_t sub[84];   // phase 0 entries, then phase 1, ...
};

struct GridCombine {
  int ch, tile, pbase, nsplit;
};

struct ChannelHost {
  std::vector<float4> geom;        // sorted order
  std::vector<int32_t> perm;       // sorted position -> original index
  std::vector<int32_t> gperm;      // gridding order -> sorted position (2x2 start blocks per sub-bin)
  std::vector<float2> vph;         // sorted order: exp(i (om_y + om_x) / 2)
  std::vector<int32_t> sb_off;     // nkeys+1
  std::vector<int64_t> block_sizes;
  int64_t M = 0;
  bool set = false;
};

struct MeasOp {
  int device = 0;
  cudaStream_t stream = nullptr;
  int Ny = 0, Nx = 0, Ky = 0, Kx = 0, Jy = 7, Jx = 7, L = 0;
  int nT0 = 0, nT1 = 0, nsb0 = 0, nsb1 = 0, nkeys = 0;
  MinMaxAxis ay, ax;
  std::vector<ChannelHost> ch;
  bool committed = false;

  // host copies of the channel layout
  std::vector<int64_t> h_voff;     // [L]
  std::vector<int32_t> h_M;        // [L]
  std::vector<int32_t> h_blkoff;   // [L] first block of each channel (global block index)
  std::vector<int32_t> h_nblk;     // [L]
  int64_t Mtot = 0;
  int nblk_tot = 0;
  int64_t maxM = 0;

  DevBuf<float2> tab_y, tab_x;
  DevBuf<float> sy, sx;
  DevBuf<float4> geom;
  DevBuf<float2> zbuf;      // pass-1 output z of the l2-ball dual update
  DevBuf<int32_t> perm;
  DevBuf<int32_t> gperm;    // [Mtot] channel-relative sorted position of the k-th visibility in gridding order
  DevBuf<float2> vph;       // [Mtot] per-visibility tap phase (sorted order)
  DevBuf<int32_t> sb_off;
  DevBuf<int64_t> ch_voff;
  DevBuf<int32_t> ch_M, ch_blkoff, ch_nblk;

  // grids: pad (FFT input, zero outside the image), A (FFT output / IFFT
  // output), B (gridding output, IFFT input).  [L][Kx][Ky] each.
  DevBuf<float2> pad, gridA, gridB;
  cufftHandle plan_all = 0, plan_one = 0;
  // real-to-complex forward path of the solvers (measop_enable_r2c): the
  // padded real image and its half spectrum (in gridA, [L][Kx][Ky/2 + 1])
  DevBuf<float> padr;
  cufftHandle plan_r2c = 0;
  // and the complex-to-real adjoint: Hermitian half of gridB (in gridA), its
  // real inverse FFT [L][Kx][Ky]
  DevBuf<float> imgr;
  cufftHandle plan_c2r = 0;
  // hand-written FFTs of the solvers' real-image path (fft.cu), for
  // power-of-two grid sides 64..4096: twiddle tables exp(-2 pi i k / K)
  // (tables built at commit when the sizes allow; own_fft: the solvers use them)
  bool own_fft = false;
  DevBuf<float2> tw_y, tw_x;
  // planes per launch of the solvers' transforms (0: all L at once); smaller
  // chunks keep each pass's intermediate in L2 for the next pass
  int fft_chunk = 0;
  // most visibilities per gridding work item (split items sum partial tiles)
  int grid_slice = 32768;
  // bumped whenever work lists or launch shapes change: solvers re-capture
  int layout_epoch = 0;
  // autotuner record (fhs_measop_autotune)
  bool tuned = false;
  std::vector<std::pair<int, double>> tune_fft, tune_grid;

  // scratch for API-level calls
  DevBuf<float2> vis_a, vis_b;
  DevBuf<double> stage;     // host-format staging (double)
  DevBuf<float> img_a;      // [L][N] image scratch
  DevBuf<double> partials;  // [degrid items][kMaxBlocksPerChannel][2]
  // work lists: channel-major items (+ per-channel offsets)
  DevBuf<WorkItem> dg_items, gr_items;
  std::vector<int> h_dg_off, h_gr_off;   // [L+1] item offsets per channel
  DevBuf<int> dg_off;                    // device copy of h_dg_off
  DevBuf<GridCombine> gr_combine;
  DevBuf<int> gr_order;                  // gridding items, largest first (whole-operator launches)
  DevBuf<GridPlan> gr_plan;              // [gridding items] sub-bin schedules
  std::vector<int> h_comb_off;           // [L+1] combine entries per channel
  DevBuf<float2> gr_partial;             // [partial slots][tile cells]
  DevBuf<double> blk_stats; // [nblk_tot][2]: ||z||^2, ||res||^2
  DevBuf<float> blk_scale;  // [L][kMaxBlocksPerChannel]
  DevBuf<double> blk_eps;   // [L][kMaxBlocksPerChannel]

  // preconditioning (set_preconditioner) and the ellipsoid projection state
  bool precond = false;
  std::vector<char> pu_set;               // [L]
  std::vector<float> h_mu;                // [L][kMaxBlocksPerChannel]
  int max_nblk = 1;                       // most blocks in any channel
  DevBuf<float> pu;                       // [Mtot] sorted order
  DevBuf<uint8_t> vblk;                   // [Mtot] block of each sorted visibility
  DevBuf<float> blk_mu;                   // [L][kMaxBlocksPerChannel]
  DevBuf<double> fb_c;                    // [L][kMaxBlocksPerChannel] scale of the next projection
  DevBuf<int> fb_iter;                    // [L][kMaxBlocksPerChannel] FB iterations done, -1 finished
  DevBuf<int> fb_count;                   // [L][kMaxBlocksPerChannel] FB iterations of the last call
  DevBuf<FbItem> fb_items;
  std::vector<int> h_fb_off;              // [L+1] FB items per channel
  DevBuf<int> fb_off;
  DevBuf<double> fb_part;                 // [fb items][kMaxBlocksPerChannel][3]

  // dimensionality reduction (visibility gridding, measop_create_dr): the
  // data space of channel c is its active grid cells W_c (diag(G^H G) > 0) in
  // column-major order; the operator is Lambda H on W_c with H = G^H G kept as
  // a half stencil T (diagonal halved, H = T + T^H) on the active cells.
  bool dr = false;
  std::vector<std::unique_ptr<DevBuf<float2>>> dr_Tc;  // [L] half stencil [kDrHalf][n_c] of the active cells
  DevBuf<float2*> dr_Tptr;  // [L] device copies of the dr_Tc pointers
  DevBuf<float2> dr_omega;  // [L][Kx][Ky] Lambda conj(rho): Lambda = diag(H)^-1/2 on W_c, 0 elsewhere
  DevBuf<int32_t> dr_map;   // [L][Kx][Ky] data index (channel-relative) of each cell, -1 off W_c
  DevBuf<int32_t> dr_cell;  // [Mtot] grid cell of each data entry
  int dr_tiles = 0;         // apply tiles per channel

  int64_t No() const { return (int64_t)Ky * Kx; }
  int64_t Npix() const { return (int64_t)Ny * Nx; }
  int ntiles() const { return nT0 * nT1; }
  OpView view() const;
  PrecondView precond_view(const double2* w) const;
  ~MeasOp();
};

MeasOp* measop_create(int device, int Ny, int Nx, int oy, int ox, int Jy, int Jx, int L);
void measop_set_channel(MeasOp* op, int channel, int64_t n, const double* om_y, const double* om_x,
                        const double* w, int n_blocks, const int64_t* block_sizes);
void measop_commit(MeasOp* op);

// ---- device building blocks used by the API and the solver -------------
// pad[l] <- s .* x[l] at (n - N/2) mod K (planes [p0, p0+np)); x: [np][N] f32
void launch_pad(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s);
// FFT of pad planes -> gridA (forward), or gridB -> gridA (inverse)
void fft_forward(const MeasOp* op, int p0, int np, cudaStream_t s);
void fft_inverse(const MeasOp* op, int p0, int np, cudaStream_t s);
// GFx for channels [c0, c0+nc) from gridA into out (sorted visibility order);
// half: gridA holds the half spectrum of fft_forward_r2c
void launch_degrid_plain(const MeasOp* op, int c0, int nc, float2* out, cudaStream_t s, bool half = false);
// real-to-complex forward path: padr <- s .* x (all planes placed as launch_pad),
// gridA <- half spectrum of padr (all L planes)
void measop_enable_r2c(MeasOp* op);
// rebuild the gridding work lists with at most `slice` visibilities per item
void measop_set_grid_slice(MeasOp* op, int slice);
// time the launch-shape candidates and keep the fastest (autotune.cu)
void measop_autotune(MeasOp* op);
void launch_pad_real(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s);
void fft_forward_r2c(const MeasOp* op, cudaStream_t s);
// imgr <- Re(IFFT(gridB)) of all L planes (Hermitian half into gridA, then C2R)
void fft_inverse_c2r(const MeasOp* op, cudaStream_t s);
// hand-written transforms (fft.cu): power-of-two grid sides 64..4096
bool measop_own_fft(const MeasOp* op);
void measop_fft_tables(MeasOp* op, cudaStream_t s);
// x: planes p0.. of the image [L][Nx][Ny] -> gridA half spectrum [L][Kx][Ky/2+1]
void fft_forward_half(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s);
// gridB [L][Kx][Ky] -> out: planes p0.. of Re(At gridB) on the image, [L][Nx][Ny], unscaled
void fft_inverse_real(const MeasOp* op, float* out, int p0, int np, cudaStream_t s);
// the solvers' real-image transforms: the hand-written ones when op->own_fft
// (imgr then holds [L][Nx][Ny]), else padr -> cuFFT R2C and C2R -> imgr [L][Kx][Ky]
void solver_fft_forward(const MeasOp* op, const float* x, cudaStream_t s);
void solver_fft_inverse(const MeasOp* op, cudaStream_t s);
// gridB <- G^H v (v sorted, channels [c0, c0+nc)); non-empty tiles only
void launch_grid_plain(const MeasOp* op, int c0, int nc, const float2* v, cudaStream_t s);
// out[l] = sigma[l] * s .* real(gridA cropped) (planes [p0, p0+np)); sigma NULL -> 1
void launch_crop_real(const MeasOp* op, float* out, const float* sigma, int p0, int np, cudaStream_t s);
// Phi x of real images x[L][Nx][Ny] (all channels) into vis (sorted order),
// and Re(Phi^H v) back into img[L][Nx][Ny]: the API-level forward / adjoint
// (hand-written FFTs when the grid sides allow them)
void measop_real_forward(const MeasOp* op, const float* img, float2* vis, cudaStream_t s);
void measop_real_adjoint(const MeasOp* op, const float2* vis, float* img, cudaStream_t s);
// img[p] *= s (the min-max scaling factors sy[iy] sx[ix]), planes [0, np) of a compact [np][Nx][Ny] image
void launch_scale_image(const MeasOp* op, float* img, int np, cudaStream_t s);
// fused dual update, pass 1: GFx, z = v2 + 2 GFx - gold - y -> zbuf, GFx -> gold, block partials
void launch_degrid_dual(const MeasOp* op, int c0, int nc, float2* v2, float2* gold, const float2* y,
                        cudaStream_t s, bool half = false);
// block reduction: scale = 1 - min(eps/||z||, 1); stats for the report
void launch_block_reduce(const MeasOp* op, int c0, int nc, cudaStream_t s);
// fused dual update, pass 2: v2 <- zbuf*scale, gridB <- G^H v2
void launch_grid_dual(const MeasOp* op, int c0, int nc, float2* v2, cudaStream_t s);

// ---- dimensionality reduction (visibility gridding, see dr.cu) ----------
// 13 x 13 coupling stencil of two 7-tap supports; its half: the diagonal and
// the 84 offsets (d0, d1) with d1 < 0 or (d1 == 0 and d0 < 0)
constexpr int kDrReach = 6;
constexpr int kDrHalf = ((2 * kDrReach + 1) * (2 * kDrReach + 1) + 1) / 2;  // 85
// builds the DR operator of a committed visibility operator (one block per
// channel); the result is committed
MeasOp* measop_create_dr(const MeasOp* vis);
// per-(channel, apply tile) partial-sum slots of the DR dual (measop_commit)
void measop_dr_lists(MeasOp* op, cudaStream_t s);
// MODE 0: out = Lambda (H Fx)(W) (gridA, half: R2C half spectrum).  MODE 1:
// l2-ball dual pass 1.  MODE 2: dual pass 2 (v2 = z scale, gridB = H Lambda v2).
// MODE 3: gridB = H (Lambda v).  (Centring phase folded in, see dr.cu.)
void launch_dr_apply(const MeasOp* op, int mode, int c0, int nc, const float2* vin, float2* out, float2* v2,
                     float2* gold, const float2* y, cudaStream_t s, bool half);

// ---- preconditioned dual (ellipsoid projection, see ellipse.cu) ---------
// pU of one channel in its original visibility order (requires a committed op)
void measop_set_preconditioner(MeasOp* op, int channel, const double* pu);
// pass 1: d = v2/pU + 2 GFx - gold - y -> zbuf, GFx -> gold, ||t_1 - y||^2 partials
void launch_degrid_dual_precond(const MeasOp* op, int c0, int nc, const float2* v2, float2* gold,
                                const float2* y, const double2* w, cudaStream_t s, bool half = false);
// block norms -> scale of the first projection, FB counters reset
void launch_block_reduce_precond(const MeasOp* op, int c0, int nc, cudaStream_t s);
// max_itr forward-backward passes (finished blocks skip their visibilities)
void launch_fb_iterations(const MeasOp* op, int c0, int nc, double2* w, const float2* y, int max_itr,
                          int min_itr, double stop, cudaStream_t s);
// pass 2: v2 = pU (d - w), gridB <- G^H v2
void launch_grid_dual_precond(const MeasOp* op, int c0, int nc, float2* v2, const double2* w, cudaStream_t s);
// w = z - y for a given z (z NULL: z = 0); z = w + y back in original visibility order (double)
void launch_w_from_proj(const MeasOp* op, const double* z_host_layout, const float2* y, double2* w,
                        cudaStream_t s);
void launch_proj_from_w(const MeasOp* op, const double2* w, const float2* y, double* z_host_layout,
                        cudaStream_t s);
// v <- sqrt(pU) .* v (root) or pU .* v (sorted order, all channels)
void launch_scale_pu(const MeasOp* op, float2* v, bool root, cudaStream_t s);
// util_gen_preconditioning_matrix, uniform weighting (host)
void gen_uniform_weights(int64_t n, const double* om_y, const double* om_x, int Ky, int Kx, int sub, double* pu);

}  // namespace fhs
