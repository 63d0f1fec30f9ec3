/*
 * subsecondpbs.h - plain C ABI of the B200 pencil-beam dose library
 * (libsubsecondpbs_b200.so).
 *
 * Every entry point takes plain pointers and sizes, so ctypes, cffi or any
 * C-compatible FFI can bind it directly. The C++ drop-in face that keeps the
 * reference's struct-based signature lives in raytracedicom_integration.h and is
 * implemented on top of these functions.
 *
 * Reference interfaces replaced (paths within Nelgcis/subsecondPBS):
 *   subsecondWrapper            include/core/raytracedicom_integration.h:132-139,
 *                               src/core/raytracedicom_wrapper.cu:2446-5661
 *   RTDBeamSettings             include/core/raytracedicom_integration.h:31-97
 *   RTDEnergyStruct             include/core/raytracedicom_integration.h:99-128
 *   cudaCalDoseRTD.raytracedicom_wrapper (pybind)
 *                               src/bindings/raytracedicom_pybind.cpp:1679-1871,2057-2086
 *
 * Error behaviour: the reference prints to stderr and returns silently on
 * invalid input (raytracedicom_wrapper.cu:1025-1157), throws std::runtime_error on
 * geometry failures (raytracedicom_wrapper.cu:3084,3177,3418) and exit(1)s on CUDA
 * errors (common.cuh:14-20). Here every failure is a non-zero status code with a
 * message available from pbs_last_error(); nothing exits the process.
 */
#ifndef SUBSECONDPBS_H
#define SUBSECONDPBS_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PBS_API __attribute__((visibility("default")))
#else
#define PBS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define PBS_OK 0
#define PBS_ERR_INVALID_ARGUMENT 1 /* input validation (reference: stderr + return) */
#define PBS_ERR_GEOMETRY 2         /* beam geometry cannot be planned (reference: throw) */
#define PBS_ERR_CUDA 3             /* CUDA runtime error (reference: exit(1)) */
#define PBS_ERR_OUT_OF_MEMORY 4    /* device allocation failed or budget exceeded */
#define PBS_ERR_UNSUPPORTED 5      /* requested mode is not available */
#define PBS_ERR_NOT_READY 6        /* context is missing CT, tables or dose grid */
#define PBS_ERR_TIMEOUT 7          /* a bounded device wait gave up */

/* ---- CT input interpretation (reference: RTD_CT_INPUT_TYPE, wrapper.cu:2280-2441) */
#define PBS_CT_AUTO 0
#define PBS_CT_HU 1
#define PBS_CT_HU_PLUS_1000 2
#define PBS_CT_DENSITY 3
#define PBS_CT_SPR 4

/* ---- context options ---------------------------------------------------- */
/* Reproduce the reference's BEV depth indexing in the per-layer transfer: the
 * reference stores BEV planes at absolute tracer steps but samples them shifted by
 * the beam's first-inside step (wrapper.cu:5308-5313 vs 5392-5394). Default 0:
 * planes are sampled where they were written (upstream RayTraceDicom behaviour). */
#define PBS_OPT_COMPAT_BEV_Z_SHIFT 1
/* Record CUDA events around each pipeline stage (read with pbs_context_stage_times). */
#define PBS_OPT_STAGE_TIMING 2
/* Device memory budget in MiB for the per-layer IDD/sigma working set (layers are
 * processed in chunks that fit). Default 2048. */
#define PBS_OPT_LAYER_BUDGET_MIB 3
/* Forced CT interpretation (PBS_CT_*); default PBS_CT_AUTO, overridden by the
 * RTD_CT_INPUT_TYPE environment variable when set. */
#define PBS_OPT_CT_INPUT_TYPE 4
/* Keep intermediate per-layer buffers of the last beam for pbs_context_debug_copy. */
#define PBS_OPT_KEEP_DEBUG 5
/* Nuclear halo model used by beams added with nuclear_correction = 1: 0 SOUKUP,
 * 1 FLUKA, 2 GAUSS_FIT (default). These are the reference's NUCLEAR_CORR build
 * choices (idd_sigma.cu:102-121, wrapper.cu:3788-3795), selected at run time here. */
#define PBS_OPT_NUCLEAR_MODEL 6
/* CarbonPBS lateral profile model of a beam's profile_data (bitmask; default 0).
 * 1: the effective sigma of every step with dose is replaced by the profile's
 * (overrideRSigmaFromCarbonProfileKernel, raytracedicom_wrapper.cu:2080-2152),
 * 2: the IDD is scaled by the profile's overall-weight channel
 * (applyCarbonProfileOverallWeightKernel, raytracedicom_wrapper.cu:2154-2187).
 * The reference compiles both but keeps them off (raytracedicom_wrapper.cu:2813-2814);
 * the wrapper entry points read PBS_CARBON_PROFILE from the environment. */
#define PBS_OPT_CARBON_PROFILE 7

/* ---- stage timer slots -------------------------------------------------- */
#define PBS_STAGE_TRACE 0
#define PBS_STAGE_PLAN 1
#define PBS_STAGE_CONV 2
#define PBS_STAGE_IDD 3
#define PBS_STAGE_BIN 4
#define PBS_STAGE_SUPERPOSE 5
#define PBS_STAGE_TRANSFER 6
#define PBS_STAGE_COUNT 7

/* ---- debug buffers (pbs_context_debug_copy) ----------------------------- */
#define PBS_DBG_DENSITY 1     /* float [steps][rayY][rayX]  BEV density            */
#define PBS_DBG_WEPL 2        /* float [steps][rayY][rayX]  cumulative WEPL (mm)   */
#define PBS_DBG_FIRST_INSIDE 3  /* int [rayY][rayX]                                */
#define PBS_DBG_FIRST_OUTSIDE 4 /* int [rayY][rayX]                                */
#define PBS_DBG_WEPL_MIN 5    /* float [steps]                                      */
#define PBS_DBG_RAY_WEIGHTS 6 /* float [layers][rayY][rayX]                         */
#define PBS_DBG_IDD 7         /* float [steps][superpY][superpX] for `layer` (0 outside [first, afterLast)) */
#define PBS_DBG_RSIGMA 8      /* float [steps][superpY][superpX] for `layer` (+inf outside)                */
#define PBS_DBG_TILE_BINS 9   /* uint8 [steps][tilesY][tilesX] for `layer`: bit7 live, bits0-6 radius bucket */
#define PBS_DBG_BEV_DOSE 10   /* float [steps][superpY+64][superpX+64], layer-summed, absolute step index */
#define PBS_DBG_DOSE64 11     /* double [Z][Y][X] accumulated dose                   */
#define PBS_DBG_FIRST_PASSIVE 12 /* int [rayY][rayX] for `layer`                    */
/* Nuclear halo of the last beam (nuclear_correction = 1), on the halo lattice
 * nucY x nucX = spot lattice rounded up to 8 x 32 (wrapper.cu:862-864). */
#define PBS_DBG_NUC_IDD 13    /* float [steps][nucY][nucX] for `layer` (0 outside [first, calcPassive)) */
#define PBS_DBG_NUC_RSIGMA 14 /* float [steps][nucY][nucX] for `layer` (+inf outside)                   */
#define PBS_DBG_NUC_TILE_BINS 15 /* uint8 [steps][nucY/8][nucX/32] for `layer` (0xff outside)          */
#define PBS_DBG_NUC_BEV_DOSE 16  /* float [steps][nucY+64][nucX+64], layer-summed, absolute step index */
#define PBS_DBG_RAY_TO_NUC 17    /* int [rayY][rayX]: halo cell under each ray or -1                  */

/* Mirrors RTDBeamSettings (include/core/raytracedicom_integration.h:31-97). Array
 * members carry their element counts (floats/ints, not rows) so the reference's
 * size validation (wrapper.cu:1099-1157) can be reproduced. NULL/0 = absent. */
typedef struct PbsBeamDesc {
    const float* energies;             size_t n_energies;              /* [L] MeV/u            */
    const float* spot_sigmas;          size_t n_spot_sigmas;           /* [L][2] sigma x,y     */
    float ray_spacing[2];
    unsigned int steps;
    float source_dist[2];
    float spot_offset[3];
    float spot_delta[3];
    int max_subspots_per_layer;
    const float* subspot_data;         size_t n_subspot_data;          /* [L][M][5]            */
    const int* layer_spot_counts;      size_t n_layer_spot_counts;     /* [L]                  */
    const float* spot_positions;       size_t n_spot_positions;        /* [N][2]               */
    int spot_positions_are_indices;
    const float* spot_weights;         size_t n_spot_weights;          /* [N]                  */
    const float* spot_beam_directions; size_t n_spot_beam_directions;  /* [N][3]               */
    const float* layer_longitudinal_cutoffs; size_t n_layer_longitudinal_cutoffs; /* [L]       */
    const float* water_equivalence;    size_t n_water_equivalence;     /* 9 header + body      */
    const float* ray_weq_header;       size_t n_ray_weq_header;        /* 9                    */
    const float* profile_data;         size_t n_profile_data;
    const float* profile_setting;      size_t n_profile_setting;
    const float* beam_para_data;       size_t n_beam_para_data;
    float beam_direction[3];
    float bm_x_direction[3];
    float bm_y_direction[3];
    float source_position[3];
    float sad;
    float ref_plane_z;
    const int* roi_linear_indices;     size_t n_roi_linear_indices;
    /* CarbonPBS lateral profile model (raytracedicom_integration.h:71-76): the
     * energy axis of the profile / beam-parameter rows (profileEnergies) and the
     * beam-parameter reference position (beamParaPos). profile_data is
     * [rows][depth][channels] (nGauss weights, nGauss sigmas, overall weight),
     * profile_setting = [depth0, depthStep, depthN], beam_para_data = [rows][3]
     * (2 sigmaIso^2, rtheta, theta^2). Used only with PBS_OPT_CARBON_PROFILE. */
    const float* profile_energies;     size_t n_profile_energies;
    float beam_para_pos;
} PbsBeamDesc;

/* Mirrors RTDEnergyStruct (include/core/raytracedicom_integration.h:99-128). */
typedef struct PbsEnergyDesc {
    int n_energy_samples;
    int n_energies;
    const float* energies_per_u;    size_t n_energies_per_u;
    const float* peak_depths;       size_t n_peak_depths;
    const float* scale_facts;       size_t n_scale_facts;
    const float* cidd_matrix;       size_t n_cidd_matrix;     /* [nEnergies][nEnergySamples] */
    int n_density_samples;
    float density_scale_fact;
    const float* density_vector;    size_t n_density_vector;
    int n_sp_samples;
    float sp_scale_fact;
    const float* sp_vector;         size_t n_sp_vector;
    int n_rrl_samples;
    float rrl_scale_fact;
    const float* rrl_vector;        size_t n_rrl_vector;
    const float* nuc_weight_matrix;   size_t n_nuc_weight_matrix;   /* [nEnergies][nEnergySamples] */
    const float* nuc_sq_sigma_matrix; size_t n_nuc_sq_sigma_matrix; /* [nEnergies][nEnergySamples] */
    int nuclear_tables_aligned_to_primary_axis;
} PbsEnergyDesc;

/* Integer/float plan of the last beam added to a context. */
typedef struct PbsBeamStats {
    int num_layers;
    int conv_mode;            /* 0 raw spot lattice (wrapper.cu:3733), 1 legacy CPB (3454) */
    int ray_dims[2];
    int superp_dims[2];
    int tracer_steps;
    int lattice_dims[2];
    float lattice_delta[2];
    float lattice_offset[2];
    float cpb_corner[2];
    float cpb_resolution[2];
    float fan_corner[3];
    float fan_delta[3];
    float source_dist[2];
    float len_to_mm;
    float energy_depth_to_mm;
    float max_peak_depth_mm;
    int first_inside;         /* beam min of per-ray first-inside step          */
    int first_outside;        /* beam max of per-ray first-outside step         */
    int guaranteed_passive;   /* min(first step past 1.05*max peak, first_outside) */
    int transfer_start[3];
    int transfer_max[3];
    long long live_tiles;     /* superposed (tile, step) pairs over all layers   */
    long long superpose_fma;  /* sum over live tiles of 256*(2R+1)^2             */
    int kernel_launches;      /* kernels this library launched for the beam      */
    int layer_chunks;         /* layer chunks the per-layer working set was split into */
    int nuc_dims[2];          /* halo lattice (0 without the nuclear halo)       */
    long long nuc_live_tiles; /* superposed halo (tile, step) pairs             */
    long long nuc_superpose_fma;
} PbsBeamStats;

typedef struct PbsLayerStats {
    float energy_idx;         /* fractional LUT row (wrapper.cu:3926-3997)       */
    float energy_scale_fact;  /* WEPL mm -> LUT depth index                      */
    float peak_depth;         /* mm                                              */
    float entry_sigma[2];     /* mm at the entry plane (wrapper.cu:3830-3833)    */
    int after_last_step;      /* wrapper.cu:4302-4304                            */
    int max_first_passive;
    int calc_passive;         /* wrapper.cu:4975-4990                            */
    int tile_rad_counts[34];  /* histogram before overflow merge                 */
    int batched_counts[33];   /* complete_superposition.cu:476-483               */
    int live_tiles;
    int nuc_tile_rad_counts[34]; /* halo histogram over [first, calc_passive)    */
    int nuc_batched_counts[33];
    float spot_dist;          /* spot spacing in rays (halo sigma and normalisation) */
} PbsLayerStats;

/* ---- library ------------------------------------------------------------ */
PBS_API const char* pbs_version(void);
PBS_API const char* pbs_last_error(void);
PBS_API int pbs_device_count(int* count);

/* One-shot pipeline with the reference's semantics: dose_data is read, the dose
 * of every beam is accumulated into it and it is written back. Host pointers. */
PBS_API int pbs_subsecond_wrapper(const float* ct_data, const int ct_dims[3], const float ct_resolution[3],
                          const float ct_corner[3], float* dose_data, const int dose_dims[3],
                          const float dose_resolution[3], const float dose_corner[3],
                          const PbsBeamDesc* beams, size_t num_beams, const PbsEnergyDesc* energy,
                          int gpu_id, int nuclear_correction, int verbose);

/* Bytes the calling thread's last completed pbs_subsecond_wrapper call moved
 * between host and device: out[0] host->device (CT box, initial dose box, tables
 * that differed from the resident ones, beam inputs, and the strided CT samples
 * the device reads from a page-locked CT for the type detection), out[1]
 * device->host (dose box, status words). No counterpart in the reference. */
PBS_API int pbs_wrapper_copy_bytes(unsigned long long out[2]);

/* Host-side planning of one beam only (no device work): validation, gantry frame,
 * spot lattice, ray grid, tracer steps and per-layer energy parameters. Fills the
 * host-known fields of `out` (device-derived fields are left 0). When
 * `layer_params` is not NULL it receives [L][8] floats per layer: energy_idx,
 * energy_scale_fact, peak_depth, conv_peak_depth, sigma_sq_air_quad,
 * sigma_sq_air_lin, sigma_x_mm, sigma_y_mm. When `lattice` is not NULL and
 * `lattice_len` equals L*ny*nx it receives the dense spot-weight lattice. */
PBS_API int pbs_plan_beam(const PbsBeamDesc* beam, const PbsEnergyDesc* energy, const int ct_dims[3],
                          const float ct_resolution[3], const float ct_corner[3], const int dose_dims[3],
                          const float dose_resolution[3], const float dose_corner[3], PbsBeamStats* out,
                          float* layer_params, float* lattice, size_t lattice_len);

/* ---- resident context (serving, benchmarking, multi-beam plans) --------- */
typedef struct PbsContext PbsContext;

PBS_API int pbs_context_create(int gpu_id, PbsContext** out);
PBS_API int pbs_context_destroy(PbsContext* ctx);
PBS_API int pbs_context_set_option(PbsContext* ctx, int option, long long value);
/* Upload the lookup tables (kept resident until replaced). */
PBS_API int pbs_context_set_energy(PbsContext* ctx, const PbsEnergyDesc* energy);
/* Upload (ct_on_device=0) or adopt a copy of (ct_on_device=1) a float CT
 * [Z][Y][X]; converted to HU+1000 on the device and kept resident. */
PBS_API int pbs_context_set_ct(PbsContext* ctx, const float* ct, int ct_on_device, const int dims[3],
                       const float resolution[3], const float corner[3]);
/* Define the dose grid; allocates the FP64 accumulator. */
PBS_API int pbs_context_set_dose_grid(PbsContext* ctx, const int dims[3], const float resolution[3],
                              const float corner[3]);
/* Reset the accumulator to `initial` (float [Z][Y][X], host or device) or to 0.
 * A host `initial` is copied on a side stream that overlaps the next beam's
 * kernels; from pinned memory the copy is asynchronous, so the buffer must stay
 * unchanged until the next add_beam, read or synchronize call has returned. */
PBS_API int pbs_context_reset_dose(PbsContext* ctx, const float* initial, int initial_on_device);
/* Plan the beam on the host and enqueue its whole pipeline on the context stream.
 * Returns without waiting for the device. */
PBS_API int pbs_context_add_beam(PbsContext* ctx, const PbsBeamDesc* beam, int nuclear_correction);
/* Spot-weight adjoint of one beam (no counterpart in the reference; the gradient
 * an inverse-planning optimiser needs). For a dose gradient G
 * (double [Z][Y][X], host or device) it writes dJ/dw_s = <G, dD/dw_s> for every
 * spot s of `beam` (n_weights floats, host, in the beam's spot order), at the
 * beam's current weights: the transposes of the transfer, the tile superposition
 * (with the forward's radii and weights), the IDD scaling and the spot -> ray
 * convolution. Dose is linear in the weights except where a ray's total weight
 * crosses the 1e-6 live threshold (idd_sigma.cu:78). Needs a raw spot lattice, no
 * nuclear halo, and every layer in one chunk (PBS_ERR_UNSUPPORTED otherwise).
 * The context's dose accumulator is not changed. Synchronous. */
PBS_API int pbs_context_adjoint_beam(PbsContext* ctx, const PbsBeamDesc* beam, const double* grad_dose,
                                     int grad_on_device, float* grad_weights, size_t n_weights);
/* Convert the accumulator to float and copy it out (host or device pointer). */
/* ---- operator mode (rtd_operator_mode.h) ---------------------------------- */
/* Mirrors RTDOperatorLayerSpan / RTDOperatorBatch (include/core/rtd_operator_mode.h:18-32). */
typedef struct PbsOperatorLayerSpan {
    int layer_index;
    int spot_begin;
    int spot_count;
    float energy;
    float longitudinal_cutoff;
} PbsOperatorLayerSpan;

typedef struct PbsOperatorBatch {
    int batch_index;
    int spot_begin;
    int spot_count;
    int first_layer_index;
    int last_layer_index;
} PbsOperatorBatch;

/* Replaces buildRTDOperatorBatchPlan (include/core/rtd_operator_mode.h:43-111).
 * info[6] = {valid, total_layers, total_spots, max_spots_per_batch, n_spans,
 * n_batches}; an invalid beam gives valid = 0 with the fields filled so far, as
 * the reference does. NULL spans/batches query the counts only; otherwise the
 * capacities must hold n_spans / n_batches (else PBS_ERR_INVALID_ARGUMENT).
 * Host only: needs no GPU. */
PBS_API int pbs_operator_batch_plan(const PbsBeamDesc* beam, int max_spots_per_batch, PbsOperatorLayerSpan* spans,
                                    int span_capacity, PbsOperatorBatch* batches, int batch_capacity, int info[6]);

/* Spot-preserving dose-influence matrix of spots [spot_begin, spot_begin +
 * spot_count) of `beam` in compressed sparse columns, the export that
 * rtd_operator_mode.h:1-8 plans and cuCalDose3 (raytracedicom_pybind.cpp:1955-2053)
 * leaves zeroed. Column j = dose per unit weight of spot spot_begin + j with the
 * beam's own plan; rows are linear voxel indices (z*Y + y)*X + x in ascending
 * order; entries with |dose| > threshold (Gy per unit weight, >= 0). Host outputs:
 * col_ptr[spot_count + 1] from 0, rows/values of `capacity` entries. *nnz is set
 * even when it exceeds `capacity`, which returns PBS_ERR_INVALID_ARGUMENT (col_ptr
 * filled, rows/values not). The beam is planned once, every spot at unit weight,
 * and each column reuses that plan with only its spot's lattice cells set. A beam
 * without a raw spot lattice (missing spot positions or weights, an empty layer, a
 * spot off the lattice phase) would run the legacy CPB fluence, which ignores
 * per-spot weights: it returns PBS_ERR_UNSUPPORTED. On return, success or error,
 * the context's dose is zero. */
PBS_API int pbs_context_influence_csc(PbsContext* ctx, const PbsBeamDesc* beam, int nuclear_correction,
                                      long long spot_begin, long long spot_count, double threshold,
                                      long long* col_ptr, int* rows, float* values, long long capacity,
                                      long long* nnz);
/* Row norms of the same influence matrix, the quantity CarbonPBS's cuCalDoseNorm
 * returns (carbonPBS/cudaCalDose.cpp:347-500, calDoseSumSquareKernel,
 * carbonPBS/deviceCalDose.cu:123-229): for every requested voxel the sum over the
 * spots [spot_begin, spot_begin + spot_count) of its squared dose per unit spot
 * weight, accumulated in FP64 on the device without forming the matrix. `voxels`
 * holds n_voxels linear indices (z*Y + y)*X + x and `out` receives one float each;
 * with voxels == NULL, `out` receives the whole grid [Z][Y][X]. Same plan, lattice
 * requirement and error behaviour as pbs_context_influence_csc; the context's dose
 * is zero on return. */
PBS_API int pbs_context_influence_row_norms(PbsContext* ctx, const PbsBeamDesc* beam, int nuclear_correction,
                                            long long spot_begin, long long spot_count, const long long* voxels,
                                            long long n_voxels, float* out);
PBS_API int pbs_context_read_dose(PbsContext* ctx, float* out, int out_on_device);
/* Copy the FP64 accumulator [Z][Y][X] out (host or device pointer), e.g. for a
 * cross-GPU reduction of beam doses. */
PBS_API int pbs_context_read_dose64(PbsContext* ctx, double* out, int out_on_device);
/* Measure the FP32 FMA throughput of `gpu_id` with a register-resident FFMA loop
 * (TFLOP/s, 2 flops per FMA): the denominator of the superposition roofline. */
PBS_API int pbs_measure_fp32_peak(int gpu_id, double* tflops);

/* ---- biological maps on top of the physical dose --------------------------
 * CarbonPBS computes, with its own point-kernel engine, the dose-averaged linear-
 * quadratic parameters of every voxel and an RBE map from them
 * (cuCalFinalDoseAndRBEKernel and LQRBEKernel, carbonPBS/deviceCalDose.cu:587-772;
 * the LEM variant lemRBEMapKernel, :1027-1057, has the same RBE arithmetic; the MKM
 * variant mkmRBEMapKernel, :1060-1126). Here the same quantities ride on this
 * library's pencil-beam dose: every step of every ray carries its IDD times the
 * step's biological factors, superposed and transferred like the dose itself.
 *
 * LET at a step: the dose-averaged LET of `let_samples` depth samples
 * t_j = LET(weq + range_shifter + (j - (n-1)/2) * est_dimension / n) of the layer's
 * energy row (let = sum t_j^2 / sum t_j, deviceCalDose.cu:686-692), from the table
 * let_table [let_rows][let_depths] (keV/um) on the depth axis let_depth0 +
 * i * let_depth_step (mm water-equivalent) and the energy axis let_energies
 * (ascending MeV/u; a layer's row is its fractional position on that axis).
 * LQ model: alpha and beta of the step from lq_alpha / lq_beta [n_lq] at
 * log10(LET) on the axis lq_log0 + i * lq_log_step (the reference's lqData is
 * indexed by log10(LET) * 100, lq_log0 = 0, lq_log_step = 0.01); the voxel mixes
 * alpha and sqrt(beta) dose-weighted. MKM: z1D [n_lq] on the same axis, mixed
 * dose-weighted, with the photon reference (alpha0, beta0). Tables are linearly
 * interpolated and clamped at their ends. Beams with the nuclear halo are refused
 * (PBS_ERR_UNSUPPORTED) while a model is set. */
#define PBS_BIO_OFF 0
#define PBS_BIO_LQ 1
#define PBS_BIO_MKM 2
typedef struct PbsBioModel {
    int model;                                    /* PBS_BIO_* */
    const float* let_table; int let_rows, let_depths;
    const float* let_energies;                    /* [let_rows] */
    float let_depth0, let_depth_step;
    int let_samples;
    float est_dimension, range_shifter;
    const float* lq_alpha;                        /* [n_lq], LQ */
    const float* lq_beta;                         /* [n_lq], LQ */
    const float* z1d;                             /* [n_lq], MKM */
    int n_lq;
    float lq_log0, lq_log_step;
    float alpha0, beta0;                          /* MKM photon reference */
} PbsBioModel;

/* Maps over the beams added since the last dose reset (an initial dose passed to
 * the reset is not part of them). DOSE: their physical dose. LETD: dose-averaged
 * LET. RBE: LQ, 3.988565 / D10 with D10 the dose of the mixed alpha, beta at 10 %
 * survival, 1 where the dose, alpha or beta is 0 (LQRBEKernel); MKM, the
 * mkmRBEMapKernel expression, 1 at or below 1e-3 Gy. RBE_DOSE: RBE x DOSE.
 * ALPHA / BETA: the mixed LQ parameters (LQ only). Z1D: 0.172 + beta0 x the mixed
 * z1D (MKM only, the reference's second MKM map). */
#define PBS_BIO_MAP_DOSE 0
#define PBS_BIO_MAP_LETD 1
#define PBS_BIO_MAP_RBE 2
#define PBS_BIO_MAP_RBE_DOSE 3
#define PBS_BIO_MAP_ALPHA 4
#define PBS_BIO_MAP_BETA 5
#define PBS_BIO_MAP_Z1D 6

/* Sets (model != PBS_BIO_OFF, tables copied to the device) or clears the model;
 * the biological accumulators start at zero and are cleared with every dose reset. */
PBS_API int pbs_context_set_bio_model(PbsContext* ctx, const PbsBioModel* model);
/* One map as float [Z][Y][X] into host (out_on_device = 0) or device memory. */
PBS_API int pbs_context_read_bio_map(PbsContext* ctx, int map, float* out, int out_on_device);

/* ---- allocation-free stage entry (no counterpart in the reference) ---------
 * Legacy CPB fluence of `n_layers` layers on the calling thread's current
 * device: subspots [n_layers][max_subspots][5] = (dx, dy, w, sigma_x, sigma_y)
 * (device memory) are integrated over the CPB cells and mapped to ray weights
 * [n_layers][ray_dims[1]][ray_dims[0]] (device memory, caller-owned, fully
 * written), as the context path does for beams without a spot lattice
 * (subspotToCPBConvolutionOptimizedKernel + mapCPBWeightsToRayWeightsKernel,
 * src/algorithms/convolution.cu:95-152, 269-339; wrapper.cu:3454-3507).
 * It exists for callers that cannot allocate device memory at the time of the
 * call (a caller-managed memory pool, a process that must not grow its
 * footprint): the CPB grid is a fixed static device array of 2^20 floats
 * (4 MiB) per device, so ray_dims[0] * ray_dims[1] * n_layers must not exceed
 * 1048576, n_layers must not exceed 65535 and ray_dims[1] not 524280 (the
 * kernels' launch limits; PBS_ERR_INVALID_ARGUMENT otherwise, before anything is
 * launched). Devices 0..63 only. No memory is allocated; the
 * scratch cells used are cleared on `stream` before use. The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress): make that first
 * call before any stream capture. The address is kept for the life of the
 * process: after a cudaDeviceReset of a device, do not call this entry point on
 * that device again. All calls on one device share the scratch, so
 * calls that overlap in time (other streams or threads) race and corrupt each
 * other's result: serialise them. Launches are asynchronous on `stream`. */
PBS_API int pbs_cpb_fluence_no_alloc(const float* d_subspots, int max_subspots, int n_layers, const int ray_dims[2],
                                     const float cpb_corner[2], const float cpb_resolution[2], float* d_ray_weights,
                                     void* stream);
PBS_API int pbs_context_synchronize(PbsContext* ctx);
/* cudaStream_t the context enqueues on. */
PBS_API void* pbs_context_stream(PbsContext* ctx);
/* Device pointer of the FP64 accumulator [Z][Y][X]. Until the pointer is handed
 * out, a zeroing reset clears only the voxels the context's beams can have
 * written and a float readout converts only those; afterwards the caller may
 * write anywhere, so every reset and readout covers the whole grid. */
PBS_API void* pbs_context_dose_device_ptr(PbsContext* ctx);
/* Stats of the last beam (synchronizes the context stream). */
PBS_API int pbs_context_beam_stats(PbsContext* ctx, PbsBeamStats* out);
PBS_API int pbs_context_layer_stats(PbsContext* ctx, int layer, PbsLayerStats* out);

/* ---- dose-request server (no reference counterpart) ------------------------
 * Continuous batching of dose requests on one GPU. `n_slots` execution slots,
 * each a resident context with its own stream and host thread, take requests
 * from one FIFO queue as they free up; a request is admitted when its device
 * bytes (tables, dose grid, largest beam) fit `hbm_budget_mib` next to the
 * resident patient CTs and the other slots (0: 90 % of the free memory). A
 * queued request that fits overtakes an older one that does not, until the older
 * one has waited `pbs_server_set_bypass_limit` seconds (default 0.5).
 * Patients are registered once: their CT is copied to pinned host memory, then
 * uploaded and converted to HU+1000 by the first request that needs it and kept
 * on the device for later requests, with the BEV traces of its beam geometries;
 * idle CTs and traces are evicted least recently used first when the budget is
 * short. Beams and tables are copied at submit and
 * registration, so the caller may free its arrays on return.
 * A result is the float [Z][Y][X] dose of the request's beams, computed as
 * pbs_context_add_beam would on a zeroed grid; `pbs_server_wait` gives a pointer
 * to it that stays valid until `pbs_server_release`. Times are seconds since the
 * server was created (submitted, started on a slot, finished). */
typedef struct PbsServer PbsServer;
typedef struct PbsServerStats {
    long long submitted, completed, failed, queued, running;
    long long patient_loads;  /* CT uploads (first use and reloads after eviction) */
    long long evictions;      /* patient CTs dropped to make room                   */
    long long slot_releases;  /* idle slots that gave their buffers back           */
    long long resident_bytes; /* patient CTs on the device                          */
    long long slot_bytes;     /* device bytes held by the slots                     */
    long long peak_bytes;     /* largest committed total at an admission            */
    long long budget_bytes;
    long long trace_hits;     /* beams that reused a resident trace                 */
    long long trace_loads;    /* traces built and kept resident                     */
    long long trace_evictions;
} PbsServerStats;

PBS_API int pbs_server_create(int gpu_id, int n_slots, long long hbm_budget_mib, PbsServer** out);
/* Stops the slots after their current request; queued requests are dropped. */
PBS_API int pbs_server_destroy(PbsServer* server);
/* PBS_OPT_COMPAT_BEV_Z_SHIFT, PBS_OPT_LAYER_BUDGET_MIB, PBS_OPT_NUCLEAR_MODEL for
 * every slot; only while no request is queued or running. */
PBS_API int pbs_server_set_option(PbsServer* server, int option, long long value);
PBS_API int pbs_server_set_bypass_limit(PbsServer* server, double seconds);
/* Resident traces (on by default): the BEV trace of a beam geometry (density,
 * WEPL, entry and exit steps) is kept per patient and reused by later beams of
 * the same geometry and tracer tables; traces count against the budget and are
 * evicted with the CTs, least recently used first. Only while idle. */
PBS_API int pbs_server_set_trace_cache(PbsServer* server, int enabled);
PBS_API int pbs_server_add_energy(PbsServer* server, int energy_id, const PbsEnergyDesc* energy);
PBS_API int pbs_server_add_patient(PbsServer* server, int patient_id, const float* ct, const int ct_dims[3],
                                   const float ct_resolution[3], const float ct_corner[3], const int dose_dims[3],
                                   const float dose_resolution[3], const float dose_corner[3]);
/* PBS_ERR_NOT_READY while a request of the patient is queued or running. */
PBS_API int pbs_server_remove_patient(PbsServer* server, int patient_id);
/* Plans every beam on the calling thread (PBS_ERR_INVALID_ARGUMENT / _GEOMETRY
 * for a beam that cannot be planned, PBS_ERR_OUT_OF_MEMORY for a request larger
 * than the budget), then queues the request. */
PBS_API int pbs_server_submit(PbsServer* server, int patient_id, int energy_id, const PbsBeamDesc* beams,
                              size_t n_beams, int nuclear_correction, unsigned long long* ticket);
/* PBS_ERR_TIMEOUT when the request is not finished within `timeout_s` (negative:
 * no limit); otherwise the request's own status. */
PBS_API int pbs_server_wait(PbsServer* server, unsigned long long ticket, double timeout_s, const float** dose,
                            double times[3], int* slot);
/* A finished request's phase times (submitted, started on a slot, all of its
 * work enqueued on the slot's stream, finished), its slot and the device bytes
 * its admission reserved on the slot. PBS_ERR_NOT_READY before it finishes. */
PBS_API int pbs_server_request_info(PbsServer* server, unsigned long long ticket, double times[4], int* slot,
                                    long long* est_bytes);
PBS_API int pbs_server_release(PbsServer* server, unsigned long long ticket);
/* Waits until nothing is queued or running. */
PBS_API int pbs_server_drain(PbsServer* server, double timeout_s);
PBS_API int pbs_server_stats(PbsServer* server, PbsServerStats* out);
PBS_API double pbs_server_now(PbsServer* server);
/* Milliseconds per stage (PBS_STAGE_*) of the last beam; needs PBS_OPT_STAGE_TIMING. */
PBS_API int pbs_context_stage_times(PbsContext* ctx, float* ms, int n);
/* Copy an intermediate buffer of the last beam (PBS_DBG_*) to host memory;
 * needs PBS_OPT_KEEP_DEBUG for the per-layer buffers. */
PBS_API int pbs_context_debug_copy(PbsContext* ctx, int which, int layer, void* host_out, size_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* SUBSECONDPBS_H */
