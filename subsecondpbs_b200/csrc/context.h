// Resident dose context (see context.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "pbs_types.h"
#include "plan.h"

namespace pbs {

void set_error(const std::string& msg);
const char* last_error();

// Grow-only device allocation; stream-ordered (cudaMallocAsync / cudaFreeAsync
// on `allocStream`) when that stream is set, so that a resize or release does not
// wait for the rest of the device.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t allocStream = nullptr;
    int ensure(size_t b);
    void release();
};

// Grow-only pinned host allocation.
struct PinnedBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t b);
    void release();
};

// Device bytes of every per-beam buffer run_beam sizes for one beam (the
// context's buffers grow to the largest beam they have run).
struct BeamBuffers {
    int chunk = 1;
    size_t dens = 0, wepl = 0, weplMin = 0, firstIn = 0, firstOut = 0, rayW = 0, bev = 0, codes = 0, work = 0, idd = 0,
           rs = 0, firstPassive = 0, lp = 0, ls = 0, bs = 0, lattice = 0, interm = 0, subspots = 0, cpb = 0;
    size_t rayToNuc = 0, nucIdd = 0, nucRs = 0, nucCodes = 0, nucWork = 0, nucBev = 0, nucLs = 0, nucBs = 0;
    size_t bevFixed = 0;  // int64 accumulator of the larger of the two BEV volumes
    size_t total(bool withTrace = true) const;
};
BeamBuffers beam_buffers(const BeamPlan& P, size_t nSubspotData, int nuclear, long long layerBudgetMiB);

struct Context;

// Where a beam's trace lives: density and WEPL [S][rays], per-ray entry and exit
// steps, the per-step WEPL minimum and the beam's first-inside / first-outside
// steps (two ints, in BeamStateDev order). A TraceStore keeps traces resident
// across beams of the same geometry; without one the context's own buffers hold
// the trace of its last beam.
struct TraceSlot {
    float* dens = nullptr;
    float* wepl = nullptr;
    int* firstIn = nullptr;
    int* firstOut = nullptr;
    float* weplMin = nullptr;
    int* inOut = nullptr;
    bool traced = false;          // holds the trace already: the tracer is skipped
    cudaEvent_t ready = nullptr;  // recorded after the trace was enqueued
};

struct TraceStore {
    virtual ~TraceStore() = default;
    // Fills `slot` for a beam of geometry `g` (dens == nullptr: not cached, use the
    // context's own buffers).
    virtual int acquire(Context& c, const BeamGeomDev& g, TraceSlot& slot) = 0;
    // The tracer into `slot` has been enqueued on the context stream.
    virtual int traced(Context& c, TraceSlot& slot) = 0;
};

// Bytes of one beam's trace (the TraceSlot arrays).
size_t trace_bytes(size_t steps, size_t rays);

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    // Host -> device copies of an initial dose run on their own stream so that they
    // overlap the beam's kernels; the FP64 grid is initialised from them just
    // before the first kernel that needs it (flush_dose_init).
    cudaStream_t copyStream = nullptr;
    cudaEvent_t copyStart = nullptr, doseCopied = nullptr;
    // Clears that no kernel needs until later in a beam run on copyStream as well:
    // the zeroing of the dose grid's dirty box (joined before anything reads or
    // rewrites the grid) and the BEV clear (joined before the superposition).
    cudaEvent_t doseZeroed = nullptr, bevCleared = nullptr;
    bool pendingDoseZero = false, pendingBevClear = false;
    bool pendingDoseInit = false;
    // The wrapper path's initial-dose box copy, issued once the beam's own uploads and
    // its trace are enqueued (issue_dose_copy) so that it does not hold them back on
    // the copy engine; the caller's buffer outlives the wrapper call.
    const float* deferredInit = nullptr;
    int deferredLo[3] = {0, 0, 0}, deferredHi[3] = {-1, -1, -1};
    // The pending initialisation covers the deferred box only (reset_dose_region).
    bool initBoxed = false;
    int issue_dose_copy();
    // While doseBoxed is set, the FP64 grid is exactly zero outside the inclusive
    // voxel box [dirtyLo, dirtyHi]: the union of the transfer boxes of the beams
    // added since the last zeroing reset. Such a reset then clears only that box,
    // and a float readout zeroes its output and converts only that box. An
    // initialised reset, a new grid or a handed-out device pointer (after which the
    // caller may write anywhere) clear the flag: the whole grid is then used.
    bool doseBoxed = false;
    bool doseExposed = false;
    int dirtyLo[3] = {0, 0, 0}, dirtyHi[3] = {-1, -1, -1};

    // Options.
    int compatBevZShift = 0;
    int stageTiming = 0;
    int keepDebug = 0;
    int ctInputType = PBS_CT_AUTO;
    long long layerBudgetMiB = 2048;
    int nuclearModel = 2;  // GAUSS_FIT
    int carbonProfile = 0; // PBS_OPT_CARBON_PROFILE bits
    int smCount = 0;       // multiprocessors of the device, read on first use

    // Lookup tables.
    bool hasEnergy = false;
    PbsEnergyDesc energy{};
    std::vector<float> energiesPerU, peakDepths, scaleFacts, ciddHost, densityHost, spHost, rrlHost;
    std::vector<float> nucWeightHost, nucSqSigmaHost;
    bool nucTablesAligned = false;
    DevBuf cidd, density, sp, rrl, nucWeight, nucSqSigma;
    DevBuf profileBuf;     // the beam's CarbonPBS profile table

    // Biological model (pbs_context_set_bio_model): tables on the device, the
    // layer rows of the current beam, the scaled IDD of one channel, the channels'
    // BEV volumes and the FP64 accumulators [4][Z][Y][X] (dose, dose x factor 0,
    // 1, 2) of the beams added since the last dose reset.
    int bioModel = 0;
    BioDev bioDev{};
    std::vector<float> bioLetEnergies;
    int bioShiftOffset[3] = {0, 0, 0};  // fixed-point exponent offset of channels 0, 1, 2
    DevBuf bioTables, bioLayerRow, bioIdd, bioBev, bioAcc;
    int set_bio_model(const PbsBioModel* m);
    int read_bio_map(int map, float* out, int onDevice);
    int clear_bio();
    LutsDev luts{};

    // CT (HU+1000) and dose accumulator.
    bool hasCt = false;
    int ctType = PBS_CT_AUTO;
    GridDesc ctGrid{};
    DevBuf ct;
    // Packed copy of `ct` for the tracer (launch_ct_quad), built by set_ct, and by
    // set_ct_region over the uploaded box; a CT attached from elsewhere is sampled
    // directly.
    DevBuf ctQuad;
    bool ctQuadValid = false;
    // A CT owned elsewhere on the same device (a server's resident patient),
    // used by the tracer in place of `ct` while set.
    const float* ctView = nullptr;
    bool hasDose = false;
    GridDesc doseGrid{};
    DevBuf dose64;

    // Per-beam working set (grow-only).
    DevBuf dens, wepl, weplMin, rayW, interm, lattice, iddBuf, rsBuf, bev, cpb, subspots, floatOut;
    DevBuf firstIn, firstOut, firstPassive, codes, work, lp, ls, bs, stats;
    // Nuclear halo working set and the device word collecting error flags.
    DevBuf rayToNuc, nucIddBuf, nucRsBuf, nucCodes, nucWork, nucBev, nucLs, nucBs, errWord;
    // Fixed-point superposition accumulator; zero between superpositions unless a
    // run stopped between a superposition and its write-out (bevFixedClean false).
    DevBuf bevFixed;
    bool bevFixedClean = false;
    BeamGeomDev nucGeom{};
    bool lastNuclear = false;
    std::vector<float> layerSpotDist;
    // Adjoint working set, and the imported water-equivalence volume of a beam.
    DevBuf gradDoseBuf, bevGrad, rbarBuf, gradInterm, gradLattice, weqBody;
    // Influence export: column offsets, per-block offsets, and the entries.
    DevBuf opColPtr, opBlockOff, opRows, opVals, opNorm, opVoxels;
    // Batched influence columns: per chunk layer (column) a BEV volume as float and as
    // int64 fixed point, and an FP64 dose buffer over colBox; all zero between
    // batches while colClean.
    DevBuf colBev, colFixed, colDose;
    ColBox colBox{};
    bool colClean = false;

    PinnedBuf staging, errHost;
    cudaEvent_t stagingEvent = nullptr;
    cudaEvent_t ev[8] = {};

    // Resident traces (a server's per-patient store), and the last beam's trace.
    TraceStore* traceStore = nullptr;
    TraceSlot trace;

    // Last beam.
    BeamPlan plan;
    BeamGeomDev geom{};
    int chunkLayers = 0;
    int lastLaunches = 0;
    int lastChunks = 0;
    bool lastBeamValid = false;
    bool lastStageTimed = false;

    ~Context();
    int init(int gpu);
    int upload(void* dst, const void* src, size_t n);
    // Bytes this context copied between host and device memory (host-visible
    // reads of a page-locked CT by the device included), for the end-to-end figures.
    unsigned long long copiedH2D = 0, copiedD2H = 0;
    int set_energy(const PbsEnergyDesc& e);
    // Reads (and clears) the error flags the kernels raised since the last check;
    // the stream must be synchronised. PBS_OK when none.
    int take_device_errors();
    // Enqueues the deferred initialisation of the FP64 grid from a host dose.
    int flush_dose_init();
    // Makes the context stream wait for the clears still running on copyStream.
    int join_side_work();
    int set_ct(const float* data, int onDevice, const GridDesc& g);
    // Wrapper path, where every beam is known before any upload: host copies limited
    // to boxes [lo, hi] (inclusive voxel indices) of the CT and of the dose grid.
    // The rest of the device CT is not read by those beams; the rest of the dose
    // grid is not written by them, so the caller's buffer keeps its values there.
    int set_ct_region(const float* data, const GridDesc& g, const int lo[3], const int hi[3]);
    // Packed CT entries of the uploaded box only (set_ct_region).
    int build_ct_quad_box(const int lo[3], const int hi[3]);
    int reset_dose_region(const float* init, const int lo[3], const int hi[3]);
    int read_dose_region(float* out, const int lo[3], const int hi[3]);
    int convert_ct(int type, const GridDesc& g);
    // HU+1000 conversion of `n` device floats in place, on the context stream.
    // With dims, only the inclusive box [lo, hi] of the [dims.z][dims.y][dims.x] CT.
    int convert_ct_buffer(float* data, size_t n, int type, const int* dims = nullptr, const int* lo = nullptr,
                          const int* hi = nullptr);
    // Per-beam buffers and the dose grid are allocated in stream order from here on.
    void use_stream_ordered_allocation();
    int set_dose_grid(const GridDesc& g);
    // Traces against a device CT (HU+1000) that the caller keeps alive.
    int attach_ct(const float* deviceCt, const GridDesc& g, int type);
    // Device bytes this context holds, and a release of the per-beam buffers and
    // the dose grid (tables and the error word stay).
    size_t device_bytes() const;
    void release_beam_buffers();
    int reset_dose(const float* init, int onDevice);
    // Adds an inclusive voxel box a beam's transfer writes to the dirty box.
    void mark_dose_written(const int lo[3], const int hi[3]);
    int read_dose(float* out, int onDevice);
    int read_dose64(double* out, int onDevice);
    int add_beam(const PbsBeamDesc& b, int nuclear);
    // add_beam with the beam's plan already made against this context's tables and
    // grids (plan_beam); the plan is moved into the context.
    int add_planned_beam(const PbsBeamDesc& b, int nuclear, BeamPlan&& planned);
    // Gradient of <gradDose, dose of the beam> with respect to the beam's spot
    // weights (one float per spot, host memory); gradDose is FP64 [Z][Y][X].
    int adjoint_beam(const PbsBeamDesc& b, const double* gradDose, int gradOnDevice, float* gradSpots, size_t nSpots);
    struct AdjointArgs {
        const double* gradDose;
        float* gradSpots;
        size_t nSpots;
    };
    // Receives the columns of a batched influence export. With a sink, every layer of
    // the plan is one column (one spot at unit weight) with its own BEV volume and
    // transfer: run_beam calls columns(first, count) once the doses of layers
    // [first, first + count) are in colDose (buffer q = layer first + q, over colBox).
    // The sink must leave those buffers zero (the compaction does). In the reference's
    // depth convention the layers are transferred one at a time into the FP64 grid
    // instead, with columns(layer, 1) after each; the sink reads and zeroes the grid.
    struct ColumnSink {
        virtual ~ColumnSink() = default;
        virtual int columns(int first, int count) = 0;
    };
    // Batched influence columns of plan P: the box every column's dose buffer is laid
    // out over, the cells of one BEV volume, and the device bytes of one column.
    void column_layout(const BeamPlan& P, ColBox& fb, size_t& bevCells, size_t& bytesPerColumn) const;
    int run_beam(const PbsBeamDesc& b, int nuclear, const AdjointArgs* adj, BeamPlan* planned = nullptr,
                 ColumnSink* cols = nullptr);
    int finish_adjoint(const AdjointArgs& a, const PbsBeamDesc& b);
    // Dose-influence columns of spots [spotBegin, spotBegin + spotCount) in CSC:
    // colPtr[spotCount + 1] (host, from 0), rows = linear voxel indices in ascending
    // order, values = dose per unit spot weight with |value| > threshold. Entries
    // past `capacity` are counted in *nnz but not copied (PBS_ERR_INVALID_ARGUMENT).
    // Leaves the dose accumulator zeroed.
    // Row norms of the influence matrix of spots [spotBegin, spotBegin + spotCount):
    // sum over the spots of each voxel's squared dose per unit weight, at the
    // voxels listed (linear indices) or, with voxels == nullptr, the whole grid.
    int influence_row_norms(const PbsBeamDesc& b, int nuclear, long long spotBegin, long long spotCount,
                            const long long* voxels, long long nVoxels, float* out);
    // Shared by the influence exports: the beam planned once at unit weights and
    // each spot's lattice cells; run_column computes one spot's dose (box: OpBox).
    struct ColumnPlan {
        std::vector<float> unit;
        PbsBeamDesc beam{};
        BeamPlan base;
        std::vector<int> cells;
        std::vector<float> shares;
    };
    int plan_columns(const PbsBeamDesc& b, long long spotBegin, long long spotCount, const char* what,
                     ColumnPlan& cp);
    // Dose of one spot at unit weight into the FP64 grid (zeroed first unless
    // `gridZero` says it is zero already), with the box of voxels it can have written.
    int run_column(ColumnPlan& cp, size_t spot, int nuclear, void* box, bool gridZero = false);
    // Doses of spots [firstSpot, firstSpot + count) at unit weight, one column at a
    // time into the FP64 grid (zeroed first unless `gridZero`), from one pass over a
    // plan with one layer per spot; sink.column(q) receives spot firstSpot + q.
    // Not for the nuclear halo, biological maps or the CarbonPBS profile model.
    int run_column_batch(ColumnPlan& cp, size_t firstSpot, int count, ColumnSink& sink, bool gridZero);
    int run_column_batches(ColumnPlan& cp, long long spotBegin, long long spotCount, int batch, ColumnSink& sink,
                           long long& first);
    int influence_csc(const PbsBeamDesc& b, int nuclear, long long spotBegin, long long spotCount, double threshold,
                      long long* colPtr, int* rows, float* vals, long long capacity, long long* nnz);
    int beam_stats(PbsBeamStats* out);
    int layer_stats(int layer, PbsLayerStats* out);
    int stage_times(float* ms, int n);
    int debug_copy(int which, int layer, void* out, size_t bytes);
};

int measure_fp32_peak(int gpu, double* tflops);

// The operator-mode batch plan of a beam (rtd_operator_mode.h:18-41).
struct OperatorPlan {
    bool valid = false;
    int totalLayers = 0;
    int totalSpots = 0;
    int maxSpotsPerBatch = 0;
    std::vector<PbsOperatorLayerSpan> spans;
    std::vector<PbsOperatorBatch> batches;
};
int operator_batch_plan(const PbsBeamDesc& beam, int maxSpotsPerBatch, OperatorPlan& plan);

// Host->device and device->host bytes of the calling thread's last completed
// subsecond_wrapper call.
int wrapper_copy_bytes(unsigned long long out[2]);
int subsecond_wrapper(const float* ctData, const int ctDims[3], const float ctRes[3], const float ctCorner[3],
                      float* doseData, const int doseDims[3], const float doseRes[3], const float doseCorner[3],
                      const PbsBeamDesc* beams, size_t numBeams, const PbsEnergyDesc* energyData, int gpuId,
                      int nuclear, int verbose);

}  // namespace pbs
