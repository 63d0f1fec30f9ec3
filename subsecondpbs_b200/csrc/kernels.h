// Kernel launchers of the dose pipeline. All launches are asynchronous on `s`.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pbs_types.h"

namespace pbs {

// ---- CT preparation -------------------------------------------------------
// Convert a float CT to HU+1000 in place according to `type` (PBS_CT_*).
cudaError_t launch_ct_convert(float* ct, size_t n, int type, const float* lut, int lutN, float lutScale,
                              cudaStream_t s);
// The same conversion over the inclusive box [lo, hi] of a [dims.z][dims.y][dims.x] CT.
cudaError_t launch_ct_convert_box(float* ct, const int dims[3], const int lo[3], const int hi[3], int type,
                                  const float* lut, int lutN, float lutScale, cudaStream_t s);
// min/max of a strided sample (the reference's ~100k-sample statistics).
cudaError_t launch_ct_stats(const float* ct, size_t n, float* minmax2, cudaStream_t s);
// The reference's ~100k-sample type detection and the conversion in one pass on
// the device: the samples are read from the caller's page-locked host CT through
// its device mapping (`hostCtMapped`, n values), the conversion runs on the
// uploaded `ct`. `keys` is two words of device scratch.
// Number of strided CT samples the type detection reads (the reference's ~100k).
size_t ct_type_sample_count(size_t n);
// CT type detection from the reference's strided samples, with the samples inside
// the uploaded box [boxLo, boxHi] read from `ct` and the others from the mapped
// host CT only when needed, then the conversion in place.
cudaError_t launch_ct_convert_detect(float* ct, size_t n, const float* hostCtMapped, const int dims[3],
                                     const int boxLo[3], const int boxHi[3], const float* densityLut, int lutN,
                                     float lutScale, unsigned* keys, cudaStream_t s);

// ---- tracing ------------------------------------------------------------------
// rayTracingBEVKernel (src/core/bev_ray_tracing.cu:65-159) as a segmented scan,
// with the per-step WEPL minimum of sliceMinVarIgnoreNeverEnter
// (src/core/raytracedicom_wrapper.cu:1991-2023) folded into its second pass.
// `ctQuad` (or null) is the packed copy of the CT from launch_ct_quad: the same
// samples from two 16-byte loads instead of eight scattered ones.
cudaError_t launch_trace(const BeamGeomDev& g, const LutsDev& luts, const float* ctHu1000, const float4* ctQuad,
                         int ctX, int ctY, int ctZ, float* density, float* wepl, int* firstInside, int* firstOutside,
                         float* weplMin, BeamStateDev* beam, cudaStream_t s);
// Packed CT for the trace: entry (x, y, z) = the HU+1000 values at (x, y), (x+1, y),
// (x, y+1), (x+1, y+1) of slice z, zero outside the CT, over a grid padded by two
// voxels below and two or three above in every axis.
size_t ct_quad_bytes(const int dims[3]);
cudaError_t launch_ct_quad(const float* ctHu1000, const int dims[3], float4* quad, cudaStream_t s);
// The packed entries of the voxels in the inclusive box [lo, hi] only (a CT uploaded
// by region: its tracers sample inside the box, two voxels in from its faces).
cudaError_t launch_ct_quad_box(const float* ctHu1000, const int dims[3], const int lo[3], const int hi[3],
                               float4* quad, cudaStream_t s);
// Beam planner: guaranteed passive step, entry plane, per-layer cut-off steps and
// entry sigmas (wrapper.cu:3651-3700, 3733-3833, 4302-4313).
// fillBevFromWeqVolumeKernel + sliceMinVarIgnoreNeverEnter (wrapper.cu:1923-2023):
// the exporter's water-equivalent depths [nx][ny][storedSteps] in place of the CT
// trace, with the per-step minimum over entering rays.
cudaError_t launch_weq_trace(const BeamGeomDev& g, const float* body, int nx, int ny, int storedSteps,
                             int activeSteps, float stepMm, float rayOriginX, float rayOriginY, float rayStepX,
                             float rayStepY, float x0, float y0, float dx, float dy, float* density, float* wepl,
                             int* firstInside, int* firstOutside, float* weplMin, BeamStateDev* beam, cudaStream_t s);
cudaError_t launch_beam_planner(const BeamGeomDev& g, float* weplMin, const LayerParamsDev* lp,
                                LayerStateDev* ls, BeamStateDev* beam, cudaStream_t s);

// ---- spot -> ray fluence ----------------------------------------------------
// x/yConvGathResampGpu (src/algorithms/convolution.cu:198-262) for all layers.
cudaError_t launch_conv_lattice(const BeamGeomDev& g, const float* lattice, float* interm, float* rayW,
                                const LayerStateDev* ls, const BeamStateDev* beam, cudaStream_t s);
// Legacy CPB fluence (convolution.cu:21-152, 269-339): subspots -> CPB -> rays.
cudaError_t launch_conv_cpb(const BeamGeomDev& g, const float* subspots, int maxSubspots, float* cpb, float* rayW,
                            cudaStream_t s);

// ---- IDD / sigma + tile radius codes -----------------------------------------
// Dynamic shared memory the IDD kernel needs (CIDD row + per-step warp partials).
size_t idd_smem_bytes(const BeamGeomDev& g, const LutsDev& luts);
// fillIddAndSigmaKernel (src/algorithms/idd_sigma.cu:46-259) fused with the
// per-tile radius reduction of tileRadCalc (complete_superposition.cu:198-255).
// With g.nucOn it also writes the nuclear halo IDD and sigma of the rays under a
// halo lattice cell (rayToNuc: [rays] -> cell or -1) into [layer][step][nucY][nucX].
cudaError_t launch_idd(const BeamGeomDev& g, const LutsDev& luts, int layer0, int nLayers, const float* density,
                       const float* wepl, const int* firstInside, const int* firstOutside, const float* rayW,
                       const LayerParamsDev* lp, LayerStateDev* ls, const BeamStateDev* beam, float* idd,
                       float* rsigma, uint8_t* codes, int* firstPassive, const int* rayToNuc, const float* lattice,
                       float* nucIdd, float* nucRsigma, cudaStream_t s);
// Histogram, overflow merge and batching (complete_superposition.cu:358-490) plus
// the radius-sorted work list of live tiles. With primaryLs/primaryBeam set it
// plans the nuclear halo grid `g` instead (no merge: a radius above 32 sets error
// flag 4). `merged` selects the forward superposition's list (items of up to
// kMergeLayers layers of one tile and step with one radius, x = the layers as bytes)
// over the one-layer items {layer | 0xffffff00, tile, step, radius} the adjoint
// gathers from, with each layer's box of live cells.
cudaError_t launch_bin_plan(const BeamGeomDev& g, int layer0, int nLayers, const uint8_t* codes, LayerStateDev* ls,
                            BeamStateDev* beam, int4* work, int workCapacity, bool merged,
                            const LayerStateDev* primaryLs, const BeamStateDev* primaryBeam, cudaStream_t s);
// Batched influence columns (one chunk layer per column, layers [0, nCols) of `ls`):
// each column's transfer box over its layer's live cells, then the transfer of BEV
// volume q (bev + q * bevStride) into dose buffer q (colDose + q * |fb|, laid out
// over fb). The BEV clear zeroes each volume's live cells afterwards.
cudaError_t launch_column_transfer(const BeamGeomDev& g, const float* bev, size_t bevStride, BeamStateDev* beam,
                                   LayerStateDev* ls, int nCols, const ColBox& fb, double* colDose, cudaStream_t s);
cudaError_t launch_column_bev_clear(const BeamGeomDev& g, float* bev, size_t bevStride, const LayerStateDev* ls,
                                    int nCols, cudaStream_t s);
// Nuclear halo: clear the chunk's halo IDD (0) and sigma (+inf) before the IDD
// kernel, and the halo tile codes and histograms after the primary layer plan.
// `gn` is the halo grid (pitch = nucX x nucY).
cudaError_t launch_nuc_prepare(const BeamGeomDev& gn, int nLayers, float* idd, float* rsigma, cudaStream_t s);
cudaError_t launch_nuc_codes(const BeamGeomDev& gn, int layer0, int nLayers, const float* idd, const float* rsigma,
                             const LayerStateDev* primaryLs, const BeamStateDev* primaryBeam, LayerStateDev* nucLs,
                             uint8_t* codes, cudaStream_t s);
// kernelSuperposition<R> (complete_superposition.cu:264-335) over the work list,
// summing all layers into one BEV dose: three persistent launches (radii 16..32,
// 8..15, 0..7) sized for `numSMs` multiprocessors accumulate the chunk in
// `bevFixed` (int64 fixed point at 2^(fixedShift + shiftOffset), all zero on entry),
// and a fifth adds it to the float `bev` and clears it again. Integer adds commute,
// so the BEV does not depend on the order in which tiles land.
cudaError_t launch_superpose(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                             BeamStateDev* beam, float* bev, unsigned long long* bevFixed, int shiftOffset,
                             int numSMs, cudaStream_t s);
// Radius blocks and claim counters of the chunk's one-layer work list
// (merged == false in launch_bin_plan), for the superposition kernels.
cudaError_t launch_one_layer_list_view(BeamStateDev* beam, cudaStream_t s);
// Batched influence columns: the chunk's whole one-layer work list (layers
// [0, nCols) of `ls`), item layer q into BEV volume q (bev / bevFixed + q * stride
// cells), each volume converted over its layer's live cells.
cudaError_t launch_superpose_columns(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                                     BeamStateDev* beam, const LayerStateDev* ls, int nCols, float* bev,
                                     unsigned long long* bevFixed, size_t stride, int numSMs, cudaStream_t s);

// ---- BEV -> dose ---------------------------------------------------------------
// Transfer bounding box and parameters (wrapper.cu:5343-5403): over the steps of
// every layer, or of `layer` alone (non-null); with `live` over the BEV cells the
// forward's superposition items can have written.
cudaError_t launch_transfer_planner(const BeamGeomDev& g, BeamStateDev* beam, const LayerStateDev* layer, int live,
                                    cudaStream_t s);
// primTransfDiv (src/algorithms/prim_transf_kernel.cu:11-44) accumulating in FP64.
cudaError_t launch_transfer(const BeamGeomDev& g, const float* bev, const BeamStateDev* beam, double* dose,
                            cudaStream_t s);

// ---- spot-weight adjoint (adjoint.cu, conv.cu) ----------------------------------------
// T^T: the dose gradient (FP64 [Z][Y][X]) spread onto the BEV gradient with the
// transfer's trilinear weights over the transfer box of `beam`.
cudaError_t launch_transfer_adjoint(const BeamGeomDev& g, const double* gradDose, const BeamStateDev* beam,
                                    float* gradBev, cudaStream_t s);
// S^T and the IDD scaling over the chunk's work list: rbar[l][ray] += idd * (S^T gradBev).
cudaError_t launch_superpose_adjoint(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                                     BeamStateDev* beam, const float* gradBev, float* rbar, int numSMs,
                                     cudaStream_t s);
// Transposed spot -> ray convolution (mode A): gradLattice[l][iy][ix] from rbar / rayW.
cudaError_t launch_conv_lattice_adjoint(const BeamGeomDev& g, const float* rbar, const float* rayW, float* gradInterm,
                                        float* gradLattice, const LayerStateDev* ls, const BeamStateDev* beam,
                                        cudaStream_t s);

// ---- dose grid -------------------------------------------------------------------
cudaError_t launch_dose_init(double* dose, const float* init, size_t n, cudaStream_t s);
cudaError_t launch_dose_to_float(const double* dose, float* out, size_t n, cudaStream_t s);
// Inclusive voxel box [lo, hi] of the dose grid: zeroes the FP64 dose there when
// `out` is null, else writes float(dose) to the same voxels of `out`.
// Inclusive box [lo, hi] of the FP64 grid initialised from the float grid `init`.
cudaError_t launch_dose_box_init(double* dose, const float* init, const int dims[3], const int lo[3], const int hi[3],
                                 cudaStream_t s);
cudaError_t launch_dose_box(double* dose, float* out, const int dims[3], const int lo[3], const int hi[3],
                            cudaStream_t s);

// Biological maps (bio.cu).
cudaError_t launch_bio_channel(const BeamGeomDev& g, const BioDev& m, int layer0, int nLayers, const float* idd,
                               const float* wepl, const LayerStateDev* ls, const BeamStateDev* beam,
                               const float* layerRow, int channel, float* out, cudaStream_t s);
cudaError_t launch_bio_map(const double* dose, const double* c0, const double* c1, const double* c2, size_t n,
                           const BioDev& m, int map, float* out, cudaStream_t s);
// Resets the superposition work list's claim counters so that the list can be run again.
cudaError_t launch_reset_work_claims(BeamStateDev* beam, cudaStream_t s);

}  // namespace pbs
