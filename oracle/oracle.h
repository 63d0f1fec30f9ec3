/*
 * CPU oracle of the pencil-beam dose path (test infrastructure only).
 *
 * A plain-C restatement of the reference pipeline behind subsecondWrapper
 * (src/core/raytracedicom_wrapper.cu:2446-5661): CT adapter, beam geometry and
 * ray grid, BEV ray tracing, beam reductions, spot->ray convolution (both fluence
 * modes), IDD/sigma, tile radius binning and batching, tile superposition and the
 * per-layer divergent transfer, and the nuclear halo branch (halo lattice IDD,
 * its own tile superposition and transfer). Geometry and every integer decision use IEEE
 * single precision in the reference's operand order (so ray grids, step counts,
 * cut-off steps, radius buckets and transfer boxes are reproduced exactly); all
 * dose arithmetic (sampling, cumulative sums, erf weights, superposition,
 * accumulation) is double precision. Layers are transferred one at a time into
 * the dose grid exactly as the reference does.
 *
 * The oracle is the checker of the CUDA library, never a fallback for it.
 */
#ifndef PBS_ORACLE_H
#define PBS_ORACLE_H

#include <stddef.h>

#include "../include/subsecondpbs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OraclePlan {
    int num_layers;
    int conv_mode;
    int ray_x, ray_y;
    int pitch_x, pitch_y;
    int tiles_x, tiles_y;
    int steps;
    int lat_nx, lat_ny;
    float lat_dx, lat_dy, lat_ox, lat_oy;
    float cpb_corner[2], cpb_res[2];
    float fan_corner[3], fan_delta[3];
    float source_dist[2];
    float len_to_mm, energy_depth_to_mm, max_peak_depth_mm;
    int bev_x, bev_y;
    int nuc_x, nuc_y;        /* halo lattice padded to 32 x 8 (0 without a spot lattice) */
    int nuc_bev_x, nuc_bev_y;
} OraclePlan;

/* Optional captures of the last beam; every pointer may be NULL. Sizes use the
 * OraclePlan of the beam (rays = ray_x*ray_y, pad = pitch_x*pitch_y,
 * tiles = tiles_x*tiles_y, S = steps, L = num_layers). */
typedef struct OracleCapture {
    double* density;        /* [S][rays]                                   */
    double* wepl;           /* [S][rays]                                   */
    int* first_inside;      /* [rays]                                      */
    int* first_outside;     /* [rays]                                      */
    double* wepl_min;       /* [S]                                         */
    int* beam_ints;         /* [4]: first_inside, first_outside, guaranteed_passive, max_calc_passive */
    double* ray_weights;    /* [L][rays]                                   */
    float* entry_sigma;     /* [L][2]                                      */
    double* idd;            /* [L][S][pad] (0 outside the computed range)  */
    double* rsigma;         /* [L][S][pad] (+inf outside)                  */
    unsigned char* codes;   /* [L][S][tiles]: bit7 live, bits0-5 bucket; 0xff outside */
    int* layer_ints;        /* [L][8]: after_last, max_first_passive, calc_passive, live_tiles, tx0,ty0,tz0 start (3) */
    int* layer_box;         /* [L][6]: transfer start xyz, max xyz        */
    int* hist;              /* [L][34] before overflow merge               */
    int* batched;           /* [L][33]                                     */
    double* bev;            /* [S][bev_y][bev_x] layer-summed, absolute step */
    double superpose_fma;   /* out: sum over live tiles of 256*(2R+1)^2     */
    /* Nuclear halo (nuclear_model >= 0), on the halo lattice nuc = nuc_x*nuc_y. */
    double* nuc_idd;        /* [L][S][nuc]                                 */
    double* nuc_rsigma;     /* [L][S][nuc] (+inf outside)                  */
    unsigned char* nuc_codes; /* [L][S][nuc tiles]                         */
    int* nuc_hist;          /* [L][34]                                     */
    int* nuc_batched;       /* [L][33]                                     */
    double* nuc_bev;        /* [S][nuc_bev_y][nuc_bev_x] layer-summed       */
    int* ray_to_nuc;        /* [rays] halo lattice cell of each ray or -1  */
    double nuc_superpose_fma;
} OracleCapture;

/* Host plan of one beam (no dose work). `layer_params` ([L][8], may be NULL)
 * receives energy_idx, energy_scale_fact, peak_depth, conv_peak_depth,
 * sigma_sq_air_quad, sigma_sq_air_lin, sigma_x_mm, sigma_y_mm. `lattice`
 * ([L][ny][nx], may be NULL, `lattice_len` floats) receives the dense spot lattice.
 * Returns PBS_OK or a PBS_ERR_* code; oracle_last_error() has the message. */
int oracle_plan(const PbsBeamDesc* beam, const PbsEnergyDesc* energy, const int ct_dims[3],
                const float ct_res[3], const float ct_corner[3], const int dose_dims[3],
                const float dose_res[3], const float dose_corner[3], OraclePlan* out, float* layer_params,
                float* lattice, size_t lattice_len);

/* Full pipeline: accumulates the dose of every beam into `dose` (double
 * [Z][Y][X], read and written). `ct_type` is a PBS_CT_* value (PBS_CT_AUTO
 * detects it as the reference does). `capture` (may be NULL) receives the
 * intermediate arrays of the last beam. `threads` <= 0 uses all cores. */
int oracle_dose(const float* ct, const int ct_dims[3], const float ct_res[3], const float ct_corner[3],
                double* dose, const int dose_dims[3], const float dose_res[3], const float dose_corner[3],
                const PbsBeamDesc* beams, size_t num_beams, const PbsEnergyDesc* energy, int ct_type,
                int compat_bev_z_shift, int threads, OracleCapture* capture);

/* The same with the nuclear halo branch: nuclear_model -1 (off), 0 SOUKUP,
 * 1 FLUKA, 2 GAUSS_FIT (the reference's NUCLEAR_CORR build values). */
int oracle_dose_nuclear(const float* ct, const int ct_dims[3], const float ct_res[3], const float ct_corner[3],
                        double* dose, const int dose_dims[3], const float dose_res[3], const float dose_corner[3],
                        const PbsBeamDesc* beams, size_t num_beams, const PbsEnergyDesc* energy, int ct_type,
                        int compat_bev_z_shift, int nuclear_model, int threads, OracleCapture* capture);

/* Tile radius bucket from a tile's minimum rSigmaEff (complete_superposition.cu:242). */
int oracle_radius_bucket(float min_rsigma);

/* Batching of a 34-bucket histogram (complete_superposition.cu:412-490): fills
 * batched[33] and map[34] (bucket -> processing radius). */
void oracle_batch(const int hist_in[34], int batched[33], int map[34]);

/* 1: quantise interpolation weights to 1/256 like the texture unit the reference
 * samples its CT, LUTs, CIDD table and BEV dose with; 0 (default): exact weights. */
void oracle_set_texture_quantization(int on);

const char* oracle_last_error(void);

/* CarbonPBS lateral profile model on the beams' profile_data (bitmask, default 0
 * as in the reference): 1 effective-sigma override, 2 overall IDD weight. */
void oracle_set_carbon_profile(int mode);

/* Biological model for the next oracle_dose calls (NULL clears it) and the
 * accumulators [4][Z][Y][X] they add to (dose, dose x factor 0, 1, 2); and the
 * maps of pbs_context_read_bio_map from such accumulators. */
void oracle_set_bio(const PbsBioModel* m, double* acc);
void oracle_bio_map(const PbsBioModel* m, const double* acc, size_t n, int map, double* out);

#ifdef __cplusplus
}
#endif

#endif /* PBS_ORACLE_H */
