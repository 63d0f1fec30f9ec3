// Structures shared between the host orchestration and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pbs_geom.h"

namespace pbs {

constexpr int kBuckets = 34;  // radius buckets 0..33 (33 = overflow, merged into 32)

// Per-layer inputs fixed by the host planner.
struct LayerParamsDev {
    float energyIdx;
    float energyScaleFact;
    float peakDepth;
    float rangeStopDepth;
    float sigmaSqAirQuad;
    float sigmaSqAirLin;
    float convPeakDepth;
    float sigmaXmm;
    float sigmaYmm;
    float spotDist;
    // CarbonPBS lateral profile model: fractional table row and beam parameters
    // (2 sigmaIso^2, rtheta, theta^2) of the layer (wrapper.cu:4577-4606).
    float profileRow;
    float bp0, bp1, bp2;
};

// Per-layer values produced on the device.
struct LayerStateDev {
    int afterLast;         // exclusive last step of the IDD loop
    float entrySigmaX;     // mm, spot->ray convolution
    float entrySigmaY;
    float entrySigmaSq;    // mm^2, IDD nuclear entry variance
    int maxFirstPassive;   // max over rays of firstPassive
    int calcPassive;       // exclusive last superposed step
    int hist[kBuckets];    // tile radius histogram over [first, calcPassive)
    int batchedR[kBuckets];     // bucket -> processing radius
    int batchedCounts[33];
    int liveTiles;
    int histAll[kBuckets];      // histogram over [first, afterLast) accumulated by the IDD kernel
    unsigned maxIddBits;        // bits of the layer's largest IDD value (non-negative floats order as ints)
    int liveHist[kBuckets];     // live tiles per raw bucket
    int liveR[33];              // live tiles per processing radius
    int offR[33];               // first work-list slot of this layer's radius-R items
    int curR[33];               // scatter cursors
    // Padded BEV cells (x, y) and steps relative to firstInside (z) this layer's
    // one-layer items (work_scatter_kernel) can write; lo > hi while none.
    int liveLo[3], liveHi[3];
    // Batched influence columns (one layer per column): the layer's own transfer box
    // over its live cells, as transfer_planner_kernel lays one out.
    int colStart[3], colMax[3], colValid;
};

// Beam-level values produced on the device.
struct BeamStateDev {
    int firstInside;        // min over rays
    int firstOutside;       // max over rays
    int guaranteedPassive;
    float entryZ;
    float pxSpMultX, pxSpMultY;
    int maxCalcPassive;
    int workCount;          // superposition work items of the current layer chunk
    // The radius-sorted work list holds the wide (R > kSplitR), medium
    // (kSplitR2 < R <= kSplitR) and narrow (R <= kSplitR2) items in that order;
    // each range has its own claim counter (relative to the range start).
    int workNext;
    int workSplit;          // items with R > kSplitR
    int workNextSmall;
    int workSplit2;         // items with R > kSplitR2
    int workNextTiny;
    // The work list holds each radius R in one block, the wide radii first; block R
    // starts at rStart[R] (layer_plan_kernel). The layer-merged list of the forward
    // superposition (work_merge_kernel) keeps mergedR[R] items at the start of R's
    // block, so the items of one radius stay together.
    int rStart[kMaxR + 1];
    int mergedR[kMaxR + 1];
    // Padded BEV cells (x, y) and steps relative to firstInside (z) the forward's
    // superposition items can write, over all chunks (work_merge_kernel); lo > hi
    // while none. The transfer box is taken over these cells.
    int liveLo[3], liveHi[3];
    // Fixed-point exponent of the chunk's BEV accumulation: a value v is added to the
    // int64 BEV as v * 2^fixedShift. Every BEV cell stays below 2^62 (layer_plan_kernel).
    int fixedShift;
    long long liveTiles;
    long long superposeFma;
    int transferStart[3];
    int transferMax[3];
    TransferParams transfer;
    int transferValid;
    int errorFlags;         // 1 work list overflow, 2 radius outside a kernel instance, 4 nuclear radius > 32
};

// Batched influence columns: the box of dose voxels (inclusive lo, extents) every
// column's dose buffer is laid out over, x fastest: the host box over the whole
// beam's transfer, which holds every layer's transfer box.
struct ColBox {
    int lo[3];
    int ext[3];
};

// The voxels a column's transfer writes: its layer's transfer box with the launch's
// block rounding in x (32) and y (8), as transfer_kernel walks a box, clipped to the
// column buffers' box. False when empty.
PBS_HD bool column_written_box(const LayerStateDev& st, int doseX, int doseY, const ColBox& fb, int lo[3],
                                      int hi[3]) {
    if (!st.colValid) return false;
    for (int i = 0; i < 3; ++i) lo[i] = st.colStart[i];
    const int nx = ((st.colMax[0] - lo[0] + 1 + 31) / 32) * 32, ny = ((st.colMax[1] - lo[1] + 1 + 7) / 8) * 8;
    hi[0] = lo[0] + (nx < doseX - lo[0] ? nx : doseX - lo[0]) - 1;
    hi[1] = lo[1] + (ny < doseY - lo[1] ? ny : doseY - lo[1]) - 1;
    hi[2] = st.colMax[2];
    bool any = true;
    for (int i = 0; i < 3; ++i) {
        if (lo[i] < fb.lo[i]) lo[i] = fb.lo[i];
        if (hi[i] > fb.lo[i] + fb.ext[i] - 1) hi[i] = fb.lo[i] + fb.ext[i] - 1;
        any = any && lo[i] <= hi[i];
    }
    return any;
}

// Everything a kernel needs to know about the beam geometry.
struct BeamGeomDev {
    TracerParams tracer;
    FromFan rayIdxToDoseIdx;
    int rayX, rayY;          // traced rays
    int pitchX, pitchY;      // superposition-padded ray grid (multiples of 32 x 8)
    int tilesX, tilesY;
    int steps;               // tracer steps
    int numLayers;
    float maxPeakDepthMm;
    V3 fanCorner, fanDelta;
    V2 sourceDist;
    float volConst, volLin, volSq;
    // Spot lattice (mode A) in gantry mm on the reference plane.
    int latNx, latNy;
    float latDx, latDy, latOx, latOy;
    float cpbCornerX, cpbCornerY, cpbResX, cpbResY;
    int bevX, bevY;          // pitch + 64
    int doseX, doseY, doseZ;
    int compatBevZShift;
    // Transport model (idd_sigma.cu:102-121): Highland reference energy, sigma
    // offset and distal-dip suppression; the GAUSS_FIT nuclear model also narrows
    // the entry sigma of the convolution (wrapper.cu:3788-3795).
    float eRefSq;
    float sigmaDelta;
    int suppressDistalDip;
    float entrySigmaScale;
    // Nuclear halo: lattice padded to 32 x 8 and the device word that collects the
    // beams' error flags until the host reads them.
    int nucOn;
    int nucX, nucY;
    int* errWord;
    // CarbonPBS lateral profile model (PBS_OPT_CARBON_PROFILE bits active for this
    // beam): table [rows][depthN][channels], its depth axis and the beam-parameter
    // position (raytracedicom_integration.h:71-76).
    int profileMode;
    const float* profile;
    int profileRows, profileDepthN, profileChannels;
    float profileDepth0, profileDepthStep;
    float beamParaPos;
};

// Biological model tables resident on the device (PbsBioModel of subsecondpbs.h).
struct BioDev {
    int model;
    const float* letTable;  // [letRows][letDepths]
    int letRows, letDepths;
    float letDepth0, letDepthStep;
    int letSamples;
    float estDimension, rangeShifter;
    const float* alpha;     // [nLq] (LQ)
    const float* beta;      // [nLq] (LQ)
    const float* z1d;       // [nLq] (MKM)
    int nLq;
    float lqLog0, lqLogStep;
    float alpha0, beta0;
};

// Lookup tables resident on the device.
struct LutsDev {
    const float* cidd;       // [nE][nS]
    int nS, nE;
    const float* density;
    int nDensity;
    float densityScale;
    const float* sp;
    int nSp;
    float spScale;
    const float* rrl;
    int nRrl;
    float rrlScale;
    const float* nucWeight;  // [nE][nS] nuclear weight, or null
    const float* nucSqSigma; // [nE][nS] nuclear sigma^2 (mm^2), or null
};

}  // namespace pbs
