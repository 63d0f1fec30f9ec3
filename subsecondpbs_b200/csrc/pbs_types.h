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
    int workNext;           // next unclaimed work item (dynamic scheduling)
    long long liveTiles;
    long long superposeFma;
    int transferStart[3];
    int transferMax[3];
    TransferParams transfer;
    int transferValid;
    int errorFlags;
};

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
};

}  // namespace pbs
