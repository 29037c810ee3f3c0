/*
 * redrock-b200: C ABI of the B200 redshift-scan engine.
 *
 * Every entry point takes plain device pointers, 64-bit sizes and a CUDA
 * stream, returns an rr_status code, and allocates no device memory: the
 * caller owns inputs, outputs and workspace (sizes are given by the
 * rr_*_workspace_bytes queries or stated per call).  Calls are asynchronous
 * on `stream`; the optional `status` argument is a device int that kernels
 * set (first error wins) when they detect bad data or a bounded wait runs
 * out, so the host can check it after synchronising.
 *
 * Reference interfaces replaced (redrock 0.22, py/redrock/...):
 *   rr_trapz_rebin          rebin.py:212-378 trapz_rebin (batch form
 *                           _trapz_rebin_batch rebin.py:178-209,
 *                           _trapz_rebin_1d rebin.py:126-176)
 *   rr_igm_transmission     igm.py:369-439 transmission_Lyman (array case;
 *                           Inoue14 igm.py:105-318, Calura12/Kamble20
 *                           igm.py:321-364)
 *   rr_build_basis          templates.py:584-597 DistTemplate.__init__
 *                           (rebin_template rebin.py:453-517 + IGM product)
 *   rr_pack_targets         zscan.py:192-209 spectral_data and
 *                           targets.py:85-89 Spectrum.Rcsr (device layout)
 *   rr_zscan_fused          zscan.py:807-889 calc_zchi2 for every template
 *                           at once (the inner loop of calc_zchi2_targets
 *                           zscan.py:910-1105), incl. calc_negOII_penalty
 *                           zscan.py:783-800
 *   rr_pack_band_rows,
 *   rr_zchi2_batch_plain    zscan.py:626-781 calc_zchi2_batch for one
 *                           target (and zscan.py:213-243 calc_zchi2_one as
 *                           nz = 1)
 *   rr_negoii_penalty       zscan.py:783-800 calc_negOII_penalty
 *   rr_pack_rows,
 *   rr_zscan_pairs          fitz.py:133-395 fine-grid refinement (every
 *                           target's own redshifts, batched)
 *   rr_zscan_pairs_grad     adjoint of the pair scan: dchi2/dz,
 *                           d2chi2/dz2, dchi2/dflux (Newton refinement in
 *                           place of fitz.py:255-261's parabola)
 *   rr_coadd, rr_coadd_ex,  targets.py:267-373 Target.compute_coadd
 *   rr_coadd_cosmics        (with cosmic-ray rejection)
 *   rr_archetype_fit        archetypes.py:228-400 archetype fits, batched
 *   rr_pack_g, rr_ygemm,    zscan.py:741-748 (y = Tb^T W f) for every
 *   rr_ygemm_i8 (+ slicing) (target, z) as one tensor-core GEMM per template
 */
#ifndef REDROCK_B200_H
#define REDROCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* same type as cudaStream_t; NULL is the legacy default stream */
typedef struct CUstream_st* rr_stream_t;

enum rr_status {
  RR_OK = 0,
  RR_EINVAL = 1,   /* bad argument (shape, pointer, unsupported layout) */
  RR_ERANGE = 2,   /* rebin edges outside the redshifted template range
                      (redrock raises ValueError, rebin.py:340-341) */
  RR_ECUDA = 3,    /* a CUDA runtime call failed; see rr_last_cuda_error */
  RR_ETIMEOUT = 4, /* a bounded device-side wait gave up */
  RR_ENOTSUP = 5,  /* valid input this build does not handle */
  RR_ESCRATCH = 6  /* request larger than rr_zchi2_batch_plain_noalloc's
                      fixed scratch (RR_NOALLOC_SCRATCH_BYTES) */
};

enum rr_igm_model { /* igm.py:367 igm_models */
  RR_IGM_NONE = 0,
  RR_IGM_CALURA12 = 1,
  RR_IGM_KAMBLE20 = 2,
  RR_IGM_INOUE14 = 3
};

enum rr_solve_method { /* zscan.py:1107-1203 solve_matrices */
  RR_SOLVE_PCA = 0,        /* linear solve; exactly singular -> HUGE_CHI2 */
  RR_SOLVE_UNSUPPORTED = 1, /* every z gets HUGE_CHI2 and zero coefficients,
                              as redrock does for NotImplementedError */
  RR_SOLVE_NNLS = 2,       /* NMF / NNLS: min ||M c - y||, c >= 0 (scipy nnls
                              on (M, y), zscan.py:1153-1169); plain path only */
  RR_SOLVE_BVLS = 3        /* min ||M c - y||, lo <= c <= hi (scipy lsq_linear
                              method='bvls', zscan.py:1170-1199); plain path
                              only (rr_zchi2_batch_plain_ex) */
};

#define RR_HUGE_CHI2 9999999.0   /* zscan.py:18 */
#define RR_HALF_BAND 5           /* resolution offsets handled: -5..5 */
#define RR_LANES 32              /* targets per target block */
#define RR_RW 12                 /* doubles per (pixel, lane): 11 band + 1 */
#ifndef RR_CHUNK
#define RR_CHUNK 24              /* pixels per scan stage */
#endif
#define RR_MAX_TEMPLATES 16
#define RR_MAX_NBASIS 10

int rr_version(void);
/* pixels per scan stage of this build: every npix_pad must be a multiple */
int rr_scan_chunk(void);
const char* rr_status_string(int status);
/* last cudaError_t seen by a call of this library on this thread */
int rr_last_cuda_error(void);

/* ------------------------------------------------------------------------
 * Trapezoidal rebinning of y(x (1+z)) onto bin edges, for every z and basis.
 *   x[nx] increasing; y[nbasis][nx]; edges[nbin+1]; z[nz]
 *   out[nz][nbin][nbasis] (the (nz, nbin, nbasis) layout redrock uses)
 * xmin/xmax/edge_min/edge_max are host copies of x[0]*(1+max z),
 * x[nx-1]*(1+min z), edges[0], edges[nbin]; RR_ERANGE if
 * edge_min < xmin or edge_max > xmax (rebin.py:330-341).  Results are bit
 * identical to redrock's CPU path for the same doubles.
 * ---------------------------------------------------------------------- */
int rr_trapz_rebin(const double* x, int64_t nx, const double* y, int64_t nbasis,
                   const double* edges, int64_t nbin, const double* z, int64_t nz,
                   double xmin, double xmax, double edge_min, double edge_max,
                   double* out, int* status, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * IGM transmission T[nz][nwave] for observed wavelengths lobs[nwave] and
 * redshifts z[nz]; model one of rr_igm_model (RR_IGM_NONE gives ones).
 * ---------------------------------------------------------------------- */
int rr_igm_transmission(int model, const double* z, int64_t nz, const double* lobs,
                        int64_t nwave, double* out, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Basis builder: rebinned (and IGM-attenuated) template for every z on the
 * union of the targets' wavelength grids, in the padded layout the scan
 * kernels read:
 *   basis[z][pix_stride][basis_stride]   (basis_stride >= nbasis, even)
 * Grid g occupies padded pixels [pix_offset - 5, pix_offset + npix_pad + 5)
 * with real pixels at [pix_offset, pix_offset + npix); everything else in
 * that range (and the basis columns >= nbasis) is written as 0.
 * ---------------------------------------------------------------------- */
typedef struct {
  const double* edges; /* device, npix + 1 */
  const double* wave;  /* device, npix pixel centres (IGM is evaluated there) */
  int64_t npix;
  int64_t npix_pad;    /* npix rounded up to a multiple of RR_CHUNK */
  int64_t pix_offset;  /* padded index of the first real pixel (>= 5) */
  double edge_min;     /* host copy of edges[0] */
  double edge_max;     /* host copy of edges[npix] */
  int apply_igm;       /* 0: skip IGM for this grid (redrock's None return) */
  int pad_;
} rr_grid_desc;

int rr_build_basis(const double* x, int64_t nx, const double* y, int64_t nbasis,
                   const double* z, int64_t nz, double xmin, double xmax,
                   const rr_grid_desc* grids /* host array */, int ngrid, int igm_model,
                   int64_t pix_stride, int basis_stride, double* basis, int* status,
                   rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Target packing for the fused scan.  Targets are grouped 32 to a block
 * (one per lane); each block walks the same list of segments (one
 * segment = one spectrum slot on one wavelength grid).  Output:
 *   rw[nblock][npix_block][12][32]: rw[.,p,k,l] = sqrt(w_p) R[p, p+k-5]
 *     (k < 11) and sqrt(w_p) f_p (k = 11) for the spectrum in (segment,
 *     lane); zero where a lane has no spectrum in that segment.
 *   fwf[nblock][32] = sum w f^2,  wsum[nblock][32] = sum w  (FP64).
 * specs are grouped by target: target t owns specs[target_first[t] ..
 * target_first[t+1]) (in redrock's spectrum order).  rw, fwf and wsum must
 * be zeroed by the caller before the call.
 * ---------------------------------------------------------------------- */
typedef struct {
  int64_t npix;        /* pixels of this spectrum */
  int64_t data_offset; /* offset of its (ndiag, npix) DIA data in rdata */
  int64_t pix_offset;  /* offset of its pixels in ivar / flux */
  int32_t ndiag;       /* diagonals stored */
  int32_t diag_offset; /* offset of its ndiag offsets in roffsets */
  int32_t block;       /* target block */
  int32_t lane;        /* lane in the block */
  int32_t segment;     /* segment index */
  int32_t pad_;
} rr_spectrum_desc;

typedef struct {
  int64_t npix_pad;     /* segment pixels rounded up to RR_CHUNK */
  int64_t basis_offset; /* padded basis index of its first pixel */
  int64_t rw_offset;    /* pixel offset of the segment in a block's rw */
} rr_segment_desc;

int rr_pack_targets(const rr_spectrum_desc* specs /* device */, int64_t nspec,
                    const int64_t* target_first /* device, ntarget + 1 */, int64_t ntarget,
                    const double* rdata, const int32_t* roffsets, const double* ivar,
                    const double* flux, const rr_segment_desc* segs /* device */, int nseg,
                    int64_t npix_block, int nblock, double* rw, double* fwf, double* wsum,
                    int* status, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Fused scan: chi2(z), coefficients(z) and the [OII] penalty for every
 * (target, template, z) in one persistent launch.
 * ---------------------------------------------------------------------- */
typedef struct {
  const double* basis;  /* [nz][pix_stride][basis_stride] from rr_build_basis */
  int64_t pix_stride;
  int32_t nz;
  int32_t nbasis;       /* 1..RR_MAX_NBASIS */
  int32_t basis_stride;
  int32_t method;       /* rr_solve_method */
  const double* prior;  /* nbasis*nbasis added to M before the solve, or NULL */
  const double* oii;    /* nbasis sums of the [OII] template window, or NULL */
  double* zchi2;        /* [nrows][nz] */
  double* zcoeff;       /* [nrows][nz][nbasis] */
  double* penalty;      /* [nrows][nz] (written only when oii != NULL) */
  const double* y_ext;  /* NULL: y = Tb^T W f is summed in the scan itself;
                           else [nblock * 32][nz][nbasis] from rr_ygemm
                           (row = block * 32 + lane) */
} rr_scan_template;

typedef struct {
  const double* rw;              /* from rr_pack_targets */
  const double* fwf;
  const double* wsum;
  const int32_t* rows;           /* [nblock][32] output row per lane, -1 empty */
  const rr_segment_desc* segs;   /* host array, nseg entries */
  int32_t nblock;
  int32_t nseg;
  int64_t npix_block;
} rr_scan_targets;

/* tile_counter: RR_FUSED_COUNTERS device ints of scratch (reset by the
 * call); on return tile_counter[2] counts the tiles that were swept a second
 * time to sum chi2 as the direct residual (ill-conditioned fits) and
 * tile_counter[3] the (target, z) pairs re-evaluated that way.  Each nbasis
 * group (10, 4, 5, any other) runs as one persistent launch with its own
 * instantiation; the launches follow one another in the stream, each after
 * the first as a programmatic dependent launch, so it starts on the SMs the
 * previous one's last tiles leave idle. */
#define RR_FUSED_COUNTERS 12
int rr_zscan_fused(const rr_scan_targets* targets, const rr_scan_template* templates,
                   int ntemplate, int* tile_counter, int* status, rr_stream_t stream);

/* Tile shape of the fused scan: a tile is 32 targets (one per lane) x 8 ZT
 * redshifts (ZT per thread, 8 warps) x 24-pixel stages.  nbasis 10 and the
 * uncommon sizes run at ZT = 1; nbasis 4 may run at ZT = 1-3 and nbasis 5
 * at ZT = 1-2 (0 = the default, 2).  block_group sets the order in which
 * the persistent CTAs take tiles: 0 = target blocks fastest (tiles running
 * at one time share basis windows); G > 0 = all redshift tiles of G target
 * blocks before the next G (their packed rows are reused while in L2).
 * Results do not depend on either choice.  rr_zscan_fused uses the
 * defaults; the host autotuner (redrock_b200/autotune.py) times the
 * choices. */
typedef struct {
  int32_t zt_nbasis4;
  int32_t zt_nbasis5;
  int32_t block_group;
} rr_scan_options;

int rr_zscan_fused_opt(const rr_scan_targets* targets, const rr_scan_template* templates,
                       int ntemplate, int* tile_counter, const rr_scan_options* opt, int* status,
                       rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Pair scan: chi2, coefficients and penalty for an arbitrary list of
 * (target, redshift) pairs, the template rebinned (+ IGM) on the fly for
 * each pair -- the batched form of fitz's fine-grid refinement
 * (fitz.py:133-395: rebin_template + transmission_Lyman + calc_zchi2_batch
 * on a 15-point grid per minimum, then a single-z fit).  Targets are packed
 * target-major by rr_pack_rows:
 *   rows[ntarget][npix_row][12] (sqrt(w) R band rows, sqrt(w) f), segment s
 *   of a target at rows[t][segs[s].rw_offset ...]; fwf[t], wsum[t].
 * Pairs whose redshift puts a bin edge outside the template range set
 * RR_ERANGE in status and get NaN outputs (check them on the host first:
 * edge_min >= x_first (1+z) and edge_max <= x_last (1+z)).
 * method RR_SOLVE_PCA solves as the fused scan does; RR_SOLVE_NNLS and
 * RR_SOLVE_BVLS (NMF templates) solve as rr_zchi2_batch_plain_ex does, with
 * chi2 the direct residual sum w (f - Tb c)^2 and HUGE_CHI2 / zero
 * coefficients where the solver fails (rr_zscan_pairs_grad: RR_ENOTSUP).
 * ---------------------------------------------------------------------- */
typedef struct {
  const double* x;      /* device, template rest wavelengths [nx] */
  int64_t nx;
  const double* y;      /* device, [nbasis][nx] */
  int32_t nbasis;
  int32_t igm_model;    /* rr_igm_model */
  int32_t method;       /* rr_solve_method */
  int32_t pad_;
  const double* prior;  /* device nbasis*nbasis or NULL */
  const double* oii;    /* device nbasis [OII] window sums or NULL */
  const double* bounds; /* HOST [2][nbasis] lower then upper bounds for
                           RR_SOLVE_BVLS (solver_args['bounds']), or NULL
                           for (-inf, inf); ignored by the other methods */
} rr_pair_template;

typedef struct {
  const double* edges;  /* device, npix + 1 bin edges of this segment's grid */
  const double* wave;   /* device, npix pixel centres */
  int64_t npix;
  int64_t row_offset;   /* pixel offset of the segment in a target's rows */
  double wave_min;      /* host copy of min(wave) */
} rr_pair_segment;

int rr_pack_rows(const rr_spectrum_desc* specs /* device */, int64_t nspec,
                 const int64_t* target_first /* device, ntarget + 1 */, int64_t ntarget,
                 const double* rdata, const int32_t* roffsets, const double* ivar,
                 const double* flux, const rr_segment_desc* segs /* device */, int nseg,
                 int64_t npix_row, double* rows, double* sw /* [ntarget][npix_row] sqrt(w),
                 or NULL */, double* fwf, double* wsum, int* status, rr_stream_t stream);

int rr_zscan_pairs(const rr_pair_template* tmpl, const rr_pair_segment* segs /* host, <= 16 */,
                   int nseg, const double* rows, const double* fwf, const double* wsum,
                   int64_t npix_row, const int32_t* pair_target, const double* pair_z,
                   int64_t npairs, double* chi2, double* coeff /* [npairs][nbasis] */,
                   double* penalty /* [npairs] or NULL */, int* status, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Adjoint of the pair scan (differentiation of chi2(z), configuration
 * "Differentiation" of this engine; redrock refines z with the parabola of
 * fitz.py:255-261 instead).  For each pair, besides chi2 (as the direct
 * residual sum), coefficients and penalty:
 *   dchi2_dz   = -2 sum_p w_p r_p (R dT/dz c)_p      (least-squares
 *                stationarity: the coefficients' own z dependence drops out)
 *   d2chi2_dz2 = 2 sum_p w_p (R dT/dz c)_p^2 - 2 (u-v)^T (M+P)^-1 (u-v)
 *                (envelope curvature without the second derivative of T;
 *                u = (R dT/dz)^T W r, v = (R T)^T W (R dT/dz c))
 *   dchi2_dflux[pair][p] = 2 w_p r_p in the packed pixel order (optional;
 *                needs sw from rr_pack_rows; not with a prior).
 *   dpenalty_dz = -oii . dc/dz where the [OII] penalty is active, else 0
 *                (optional), with dc/dz = (M+P)^-1 (u-v): the derivative of
 *                the objective fitz minimises, chi2 + penalty, is
 *                dchi2_dz + dpenalty_dz.
 * dT/dz is exact for the trapezoid rebin (from the bin-edge values of the
 * redshifted interpolant) and includes the smooth z dependence of the
 * Inoue14 Lyman-continuum optical depth; on/off switches of IGM lines with z
 * are steps with no derivative.
 * ---------------------------------------------------------------------- */
int rr_zscan_pairs_grad(const rr_pair_template* tmpl, const rr_pair_segment* segs, int nseg,
                        const double* rows, const double* sw, const double* fwf,
                        const double* wsum, int64_t npix_row, const int32_t* pair_target,
                        const double* pair_z, int64_t npairs, double* chi2, double* coeff,
                        double* penalty, double* dchi2_dz, double* d2chi2_dz2,
                        double* dchi2_dflux, double* dpenalty_dz, int* status,
                        rr_stream_t stream);

/* ------------------------------------------------------------------------
 * fitz candidates on the device: replaces the host steps of redrock's fitz
 * between the coarse scan and the fine-grid evaluations --
 * find_minima (fitz.py:46-67: local minima with <= comparisons, edges
 * included, sorted by value) and the fine grids
 * zz = np.linspace(z[i-1], z[i+1], nfine) (fitz.py:226-240, indices clipped)
 * -- so that the scan and the fine-grid pair scans (rr_zscan_pairs on
 * pair_t / pair_z) run without a host round trip.  Per target row of
 * zchi2 + penalty ([ntarget][nz]; penalty may be NULL): the K (<= 8)
 * smallest minima in cand[ntarget][K] (-1 past count[t]), tie[t] = 1 when
 * equal values make redrock's (unstable) sort order undetermined -- sort
 * those rows on the host -- and pair_z / pair_t [ntarget][K][nfine], the
 * fine grid of each candidate (slots past count repeat candidate 0).
 * ---------------------------------------------------------------------- */
int rr_fitz_candidates(const double* zchi2, const double* penalty, int64_t ntarget, int64_t nz,
                       const double* redshifts, int32_t K, int32_t nfine, int32_t* cand,
                       int32_t* count, int8_t* tie, double* pair_z, int32_t* pair_t,
                       rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Plain per-target path (the structure of redrock's own GPU branch: R.T for
 * all z into a workspace, then M and y, then the solve, then the model and
 * chi2).  First pack the target's spectra into band rows:
 *   band[P][11], w[P], wflux[P], flux[P]  (P = sum of spectrum pixels, in
 *   spectrum order) and seg_basis[P]: padded basis index of each pixel.
 * ---------------------------------------------------------------------- */
int rr_pack_band_rows(const rr_spectrum_desc* specs /* device */, int64_t nspec,
                      const double* rdata, const int32_t* roffsets, int64_t npix_total,
                      double* band, int* status, rr_stream_t stream);

/* Workspace bytes of one call; SIZE_MAX when the count overflows (every
 * size check against it then fails with RR_EINVAL / RR_ESCRATCH). */
size_t rr_zchi2_batch_plain_workspace_bytes(int64_t npix_total, int32_t nz, int32_t nbasis);

/* rr_zchi2_batch_plain with the bounds of RR_SOLVE_BVLS: a host array
 * [2][nbasis] (lower row, then upper; +-INFINITY allowed) or NULL for
 * (-inf, inf) -- redrock's solver_args['bounds'].  For RR_SOLVE_NNLS and
 * RR_SOLVE_BVLS chi2 is the direct residual sum w (f - Tb c)^2 (as for
 * every method of this path); a failed bounded solve (singular free set,
 * iteration limit) gives HUGE_CHI2 like redrock's caught exception.
 * status (optional): RR_EINVAL when a pix_basis entry puts its 11-row band
 * outside the basis rows [0, pix_stride) (those pixels read nothing and
 * count as zero model); check it before trusting the outputs. */
int rr_zchi2_batch_plain_ex(const double* band, const double* w, const double* wflux,
                            const double* flux, const int64_t* pix_basis, int64_t npix_total,
                            const double* basis, int64_t pix_stride, int32_t nz, int32_t nbasis,
                            int32_t basis_stride, const double* prior, int32_t method,
                            const double* bounds, double* zchi2, double* zcoeff, void* workspace,
                            size_t workspace_bytes, int* status, rr_stream_t stream);

int rr_zchi2_batch_plain(const double* band, const double* w, const double* wflux,
                         const double* flux, const int64_t* pix_basis, int64_t npix_total,
                         const double* basis, int64_t pix_stride, int32_t nz, int32_t nbasis,
                         int32_t basis_stride, const double* prior, int32_t method,
                         double* zchi2, double* zcoeff, void* workspace, size_t workspace_bytes,
                         int* status, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * rr_zchi2_batch_plain without a caller-provided workspace.  No counterpart
 * in redrock.  For callers that cannot allocate device memory themselves --
 * programs whose own memory manager already owns the GPU's memory, or
 * latency-bound loops in which cudaMalloc / cudaFree could synchronise the
 * device -- it works in a fixed scratch array compiled into the library
 * (every GPU that loads the library holds RR_NOALLOC_SCRATCH_BYTES until
 * exit) and allocates nothing.  Requests with
 * rr_zchi2_batch_plain_workspace_bytes(npix_total, nz, nbasis) >
 * RR_NOALLOC_SCRATCH_BYTES return RR_ESCRATCH.  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * The first call on a device looks up the array's address and caches it;
 * make it before any stream capture, and do not use this entry point again
 * after cudaDeviceReset on that device (the cached address is stale).
 * ---------------------------------------------------------------------- */
#define RR_NOALLOC_SCRATCH_BYTES (16u << 20)

int rr_zchi2_batch_plain_noalloc(const double* band, const double* w, const double* wflux,
                                 const double* flux, const int64_t* pix_basis,
                                 int64_t npix_total, const double* basis, int64_t pix_stride,
                                 int32_t nz, int32_t nbasis, int32_t basis_stride,
                                 const double* prior, int32_t method, double* zchi2,
                                 double* zcoeff, int* status, rr_stream_t stream);

/* penalty[z] = max(0, -sum_b coeff[z][b] oii[b])  (zscan.py:783-800) */
int rr_negoii_penalty(const double* coeff, int64_t nz, int32_t nbasis, const double* oii,
                      double* penalty, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Tensor-core y (zscan.py:741-748, y = Tb^T W f) for the fused scan.
 * y_i(t, z) = sum_q G[q][t] T_z[q][i] with G[., t] = R^T W f of target t
 * (independent of z), so y of a whole template is one GEMM
 * (targets x pixels) . (pixels x (z, basis)) run on tcgen05:
 *   RR_YGEMM_BF16X3  three bf16 slices, six products, FP32 accumulation
 *   RR_YGEMM_TF32X3  two tf32 slices, three products, FP32 accumulation
 *   RR_YGEMM_INT8X7  Ozaki scheme: each G column / basis column scaled by a
 *                    power of two and rounded to a 49-bit integer of seven
 *                    base-128 digits; the 28 digit products of order <= 6
 *                    accumulate exactly in int32 and combine in FP64
 *                    (error <= K 2^-45 2^(e_t + e_n) per output); K <= 65536
 *   RR_YGEMM_INT8X6  the same with six base-256 digits of a 48-bit integer
 *                    (|X| <= 127 2^40): 21 products of order <= 5, 80 output
 *                    columns per tile instead of 64 (error <= K 2^-44
 *                    2^(e_t + e_n)); K <= 21824
 * Flow: rr_pack_targets -> rr_pack_g (G, row_exp) -> per template
 *   BF16X3 / TF32X3: rr_ygemm
 *   INT8X7 / INT8X6: rr_slice_g_i8 (once per target pack), rr_basis_col_exp
 *           + rr_slice_basis_i8 (once per basis), rr_ygemm_i8
 * -> rr_zscan_fused with y_ext = Y.
 * ---------------------------------------------------------------------- */
enum rr_ygemm_variant {
  RR_YGEMM_NONE = 0,   /* y summed in FP64 inside the scan (default) */
  RR_YGEMM_BF16X3 = 1,
  RR_YGEMM_TF32X3 = 2,
  RR_YGEMM_INT8X7 = 3,
  RR_YGEMM_INT8X6 = 4
};

/* padded pixel count (rows of G) for a basis of pix_stride rows */
int64_t rr_ygemm_kpad(int64_t pix_stride);

/* G[kpad][npos] (row q = padded basis pixel, column = block * 32 + lane)
 * and row_exp[npos] (biased power-of-two exponents e of each column with
 * max |G| < 127/128 2^e <= 2 max |G|, or NULL).  npos: a multiple of 128, >= nblock * 32.  The call zeroes G
 * and row_exp first. */
int rr_pack_g(const rr_scan_targets* targets, int64_t pix_stride, int64_t kpad, int64_t npos,
              double* g, int* row_exp, int* status, rr_stream_t stream);

/* col_exp[nz * nbasis]: biased exponent e of max_q |basis[z][q][i]| with
 * the same 127/128 margin */
int rr_basis_col_exp(const double* basis, int64_t nz, int64_t pix_stride, int nbasis,
                     int basis_stride, int* col_exp, rr_stream_t stream);

/* y[npos][nz][nbasis] = G^T . basis, variant RR_YGEMM_BF16X3 or _TF32X3 */
int rr_ygemm(int variant, const double* g, int64_t npos, int64_t kpad, const double* basis,
             int64_t nz, int64_t pix_stride, int nbasis, int basis_stride, double* y,
             int* status, rr_stream_t stream);

/* RR_YGEMM_INT8X7 / RR_YGEMM_INT8X6 (variant): digit planes of G and of a
 * basis, laid out as the GEMM's shared-memory tiles (16-byte aligned
 * buffers of the sizes returned by the _bytes queries, -1 for invalid
 * arguments); digits and GEMM must use the same variant */
int64_t rr_ygemm_i8_g_bytes(int variant, int64_t npos, int64_t kpad);
int64_t rr_ygemm_i8_basis_bytes(int variant, int64_t nz, int nbasis, int64_t kpad);
/* largest kpad whose int32 accumulation stays exact (-1: not an INT8 variant) */
int64_t rr_ygemm_i8_max_kpad(int variant);
int rr_slice_g_i8(int variant, const double* g, const int* row_exp, int64_t npos, int64_t kpad,
                  void* g_digits, rr_stream_t stream);
int rr_slice_basis_i8(int variant, const double* basis, int64_t nz, int64_t pix_stride,
                      int nbasis, int basis_stride, int64_t kpad, const int* col_exp,
                      void* basis_digits, rr_stream_t stream);
/* y[npos][nz][nbasis]; RR_ENOTSUP when kpad > rr_ygemm_i8_max_kpad(variant) */
int rr_ygemm_i8(int variant, const void* g_digits, const int* row_exp, int64_t npos,
                int64_t kpad, const void* basis_digits, const int* col_exp, int64_t nz,
                int nbasis, double* y, int* status, rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Coadd of a target's exposures per wavelength grid (targets.py:267-373,
 * Target.compute_coadd).  Per group of nspec
 * exposures (entries first .. first + nspec - 1 of exp_data / exp_pix):
 *   ivar_out  = sum ivar;  flux_out = sum ivar flux / sum ivar (sum flux /
 *   nspec where sum ivar == 0);  rdata_out[d] = sum data[d] ivar / sum ivar
 *   (/ 1 where 0), DIA data column-indexed, all sums in exposure order, so
 * the results are bit-identical to redrock's numpy.  exp_data[e] / exp_pix[e]
 * are offsets of exposure e's (ndiag, npix) data in rdata and its pixels in
 * ivar / flux.  ngroup <= 65535; max_npix = largest group npix.
 * ---------------------------------------------------------------------- */
typedef struct {
  int64_t npix;
  int32_t ndiag;
  int32_t nspec;     /* exposures in the group (>= 1) */
  int64_t first;     /* first exposure index of the group */
  int64_t out_pix;   /* offset of the group's pixels in ivar_out / flux_out */
  int64_t out_data;  /* offset of its (ndiag, npix) data in rdata_out */
} rr_coadd_group;

int rr_coadd(const rr_coadd_group* groups /* device */, int64_t ngroup, int64_t max_npix,
             const int64_t* exp_data, const int64_t* exp_pix, const double* rdata,
             const double* ivar, const double* flux, double* rdata_out, double* ivar_out,
             double* flux_out, rr_stream_t stream);
/* rr_coadd with the resolution data weighted by ivar_rdata (NULL = ivar):
 * after cosmic-ray rejection redrock weights R by the exposures' own ivar
 * and the flux by the masked one (targets.py:300-301 vs 356-358). */
int rr_coadd_ex(const rr_coadd_group* groups, int64_t ngroup, int64_t max_npix,
                const int64_t* exp_data, const int64_t* exp_pix, const double* rdata,
                const double* ivar_rdata, const double* ivar, const double* flux,
                double* rdata_out, double* ivar_out, double* flux_out, rr_stream_t stream);
/* Cosmic-ray rejection of compute_coadd(cosmics_nsig > 0), targets.py:310-354:
 * ivar_out (layout of ivar, npix_total values) = ivar with the outlier
 * pixels of groups of >= 2 exposures set to 0, bit-identical to redrock.
 * wave holds each group's wavelengths at its out_pix offset; nsig2 =
 * cosmics_nsig**2; work = 2 * npix_total doubles.  An exposure without a
 * pixel of ivar > 0 sets *status = RR_EINVAL (numpy raises ValueError). */
int rr_coadd_cosmics(const rr_coadd_group* groups, int64_t ngroup, const int64_t* exp_pix,
                     const double* wave, const double* ivar, const double* flux, double nsig2,
                     double* ivar_out, double* work, int64_t npix_total, int* status,
                     rr_stream_t stream);

/* ------------------------------------------------------------------------
 * Archetype fits for many (target, redshift) pairs at once
 * (archetypes.py:228-400: Archetype.get_best_archetype /
 * nearest_neighbour_model, whose solves are calc_zchi2_batch and
 * per_camera_coeff_with_least_square_batch, zscan.py:245-348, 626-781).
 *
 * Pair i: the target's pixels pix_off .. pix_off + npix - 1 of the
 * concatenated band rows (npix x 11, row p multiplies basis rows
 * pix_basis[p] - 5 .. + 5, as rr_pack_band_rows writes them), w, wflux =
 * w f and flux; its archetype columns arch[arch_off + a * pix_stride + row]
 * (a < narch: rebinned x IGM, zero outside the grids) and nl Legendre
 * columns leg[leg_off + k * pix_stride + row].  Job j of pair i fits the m
 * archetypes jobs[(i * njob + j) * m ..] followed by the nl Legendre
 * columns: nb = m + nl <= RR_MAX_NBASIS coefficients solved from
 * (Tb^T W Tb + prior) c = Tb^T W f with method RR_SOLVE_PCA / NNLS / BVLS
 * (bounds: host [2][nb], NULL = unbounded), chi2 = sum w (f - Tb c)^2 (the
 * prior excluded).  Outputs chi2[i * njob + j] and coeff[(i * njob + j) *
 * nb ..]; a failed solve or an archetype index outside [0, narch) gives
 * RR_HUGE_CHI2 and zero coefficients.  prior: device nb x nb or NULL.
 * ---------------------------------------------------------------------- */
typedef struct {
  int64_t pix_off;
  int64_t npix;
  int64_t arch_off;
  int64_t leg_off;
} rr_arch_pair;

/* work: device scratch of rr_archetype_fit_work_bytes(npair, njob, m, nl, max_npix),
 * max_npix >= every pair's npix (R L of each pair's Legendre columns is
 * built once there and shared by the pair's jobs) */
size_t rr_archetype_fit_work_bytes(int64_t npair, int32_t njob, int32_t m, int32_t nl,
                                   int64_t max_npix);
int rr_archetype_fit(const rr_arch_pair* pairs /* device */, int64_t npair, const double* band,
                     const int64_t* pix_basis, const double* w, const double* wflux,
                     const double* flux, int64_t max_npix, const double* arch, int32_t narch,
                     const double* leg, int64_t pix_stride, const int32_t* jobs, int32_t njob,
                     int32_t m,
                     int32_t nl, const double* prior, int32_t method, const double* bounds,
                     double* chi2, double* coeff, void* work, size_t work_bytes,
                     rr_stream_t stream);

/* ------------------------------------------------------------------------
 * FMA throughput probe (no counterpart in redrock): the roofline
 * denominator of the FP64-bound scan.  kind 0 = FP64, 1 = FP32; issues
 * 2*8*16*iters*blocks*256 FLOPs; out is one device element of that type.
 * ---------------------------------------------------------------------- */
int rr_fma_peak(int kind, int blocks, int iters, void* out, rr_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* REDROCK_B200_H */
