// Dose-request server: continuous batching of dose requests over a fixed set of
// execution slots on one GPU, with per-patient CT kept resident in HBM under a
// byte budget.
//
// A slot is a resident Context (its own stream, tables, per-beam buffers and FP64
// dose grid) driven by its own host thread. Requests wait in one FIFO queue; a
// slot that becomes free takes the first queued request whose device bytes fit
// the budget next to everything already resident or running (a request that has
// waited longer than `maxBypassSec` blocks the ones behind it from overtaking).
// Patients' CTs are uploaded once (from a pinned host copy made at registration),
// converted to HU+1000 on the device, and shared read-only by every slot; when the
// budget is short, idle patients are evicted least recently used first, then idle
// slots give their buffers back. All device allocations of the server are
// stream-ordered, so resizing one slot never waits for the others.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/subsecondpbs.h"
#include "context.h"

namespace pbs {

// Deep copy of a beam descriptor (the caller may free its arrays after submit).
struct OwnedBeam {
    PbsBeamDesc d{};
    std::vector<float> energies, sigmas, subspots, positions, weights, directions, cutoffs, weq, weqHeader, profile,
        profileSetting, beamPara;
    std::vector<int> counts, roi;
    void assign(const PbsBeamDesc& b);
};

// Deep copy of the lookup tables; `lutHash` identifies the HU -> density and
// stopping-power tables the tracer uses.
struct OwnedEnergy {
    PbsEnergyDesc d{};
    std::vector<float> energiesPerU, peakDepths, scaleFacts, cidd, density, sp, rrl, nucWeight, nucSqSigma;
    unsigned long long lutHash = 0;
    void assign(const PbsEnergyDesc& e);
};

struct Request;

// A beam geometry's trace kept resident for one patient (see TraceSlot).
struct TraceEntry {
    size_t bytes = 0;
    void* mem = nullptr;
    TraceSlot slot;
    enum State { Absent, Loading, Ready } state = Absent;
    cudaEvent_t ready = nullptr;
    int pins = 0;
    unsigned long long lastUse = 0;
    const Request* loader = nullptr;
};

struct Patient {
    int id = 0;
    GridDesc ctGrid{}, doseGrid{};
    int ctType = PBS_CT_AUTO;
    PinnedBuf hostCt;               // the CT as registered
    void* deviceCt = nullptr;       // HU+1000 on the device while resident
    size_t ctBytes = 0;
    enum State { Absent, Loading, Resident } state = Absent;
    cudaEvent_t ready = nullptr;    // recorded after the upload and conversion
    int pins = 0;                   // admitted requests using the CT
    unsigned long long lastUse = 0;
    int loads = 0;
    std::map<std::string, std::unique_ptr<TraceEntry>> traces;  // by trace_key
};

struct Request {
    unsigned long long ticket = 0;
    int patientId = 0, energyId = 0, nuclear = 0;
    Patient* patient = nullptr;
    std::vector<OwnedBeam> beams;
    const OwnedEnergy* energy = nullptr;
    std::vector<std::string> traceKeys;   // per beam
    std::vector<size_t> traceBytes;
    std::vector<TraceEntry*> traces;      // pinned at admission
    size_t estBytes = 0;            // slot bytes the request needs (tables, dose grid, largest beam)
    bool loadsPatient = false;      // admitted while the patient's CT was absent
    double tSubmit = 0, tStart = 0, tEnqueued = 0, tDone = 0;
    int slot = -1;
    int state = 0;                  // 0 queued, 1 running, 2 done
    int rc = PBS_OK;
    std::string error;
    PinnedBuf result;               // float [Z][Y][X] dose of the request
};

class Server;

// The slot's view of the server's resident traces (Context::traceStore).
struct SlotTraces : TraceStore {
    Server* server = nullptr;
    struct Slot* slot = nullptr;
    int acquire(Context& c, const BeamGeomDev& g, TraceSlot& ts) override;
    int traced(Context& c, TraceSlot& ts) override;
};

struct Slot {
    int index = 0;
    Context ctx;
    SlotTraces traces;
    std::thread thread;
    Request* current = nullptr;
    size_t bytes = 0;               // device bytes the slot's context holds (updated between requests)
};

struct ServerStats {
    long long submitted = 0, completed = 0, failed = 0, queued = 0, running = 0;
    long long patientLoads = 0, evictions = 0, slotReleases = 0;
    long long traceHits = 0, traceLoads = 0, traceEvictions = 0;
    size_t residentBytes = 0, slotBytes = 0, peakBytes = 0, budgetBytes = 0;
};

class Server {
   public:
    ~Server();
    int init(int gpu, int nSlots, size_t budgetBytes);
    int set_option(int option, long long value);
    int set_trace_cache(bool on);
    int add_energy(int id, const PbsEnergyDesc& e);
    int add_patient(int id, const float* ct, const GridDesc& ctGrid, const GridDesc& doseGrid);
    int remove_patient(int id);
    int submit(int patientId, int energyId, const PbsBeamDesc* beams, size_t nBeams, int nuclear,
               unsigned long long* ticket);
    // Waits up to `timeoutSec` (negative: no limit) for the request; on success
    // `dose` points at its float [Z][Y][X] result, valid until release().
    int wait(unsigned long long ticket, double timeoutSec, const float** dose, double times[3], int* slot);
    // Phase times of a finished request: submitted, started on a slot, all of its
    // work enqueued, finished; and its slot and device-byte estimate.
    int info(unsigned long long ticket, double times[4], int* slot, long long* estBytes);
    int release(unsigned long long ticket);
    int drain(double timeoutSec);
    void stats(ServerStats* out);
    double now() const;

    double maxBypassSec = 0.5;
    bool traceCache = true;

    int trace_acquire(Slot& s, const BeamGeomDev& g, TraceSlot& ts);
    int trace_done(Slot& s, TraceSlot& ts);

   private:
    void worker(Slot* s);
    Request* pick(Slot& s);                       // mu held
    bool make_room(size_t need, const Request& r, Slot& s);  // mu held
    void evict_trace(TraceEntry& e, cudaStream_t s);      // mu held
    size_t committed_bytes() const;               // mu held
    int execute(Slot& s, Request& r);
    int ensure_resident(Slot& s, Request& r);
    int acquire_result(Request& r, size_t bytes);
    void recycle_result(PinnedBuf& b);

    int device_ = 0;
    size_t budget_ = 0;
    std::chrono::steady_clock::time_point t0_;
    std::vector<std::unique_ptr<Slot>> slots_;
    std::map<int, std::unique_ptr<OwnedEnergy>> energies_;
    std::map<int, std::unique_ptr<Patient>> patients_;
    std::map<unsigned long long, std::unique_ptr<Request>> requests_;
    std::deque<Request*> queue_;
    std::multimap<size_t, void*> freeResults_;
    std::mutex mu_, poolMu_;
    std::condition_variable cvWork_, cvDone_, cvLoad_;
    bool stopping_ = false;
    unsigned long long nextTicket_ = 1, useClock_ = 0;
    size_t residentBytes_ = 0, peakBytes_ = 0;
    long long submitted_ = 0, completed_ = 0, failed_ = 0, running_ = 0, loads_ = 0, evictions_ = 0,
              slotReleases_ = 0, traceHits_ = 0, traceLoads_ = 0, traceEvictions_ = 0;
    long long layerBudgetMiB_ = 2048;
    int nuclearModel_ = 2, compatBevZShift_ = 0;
};

}  // namespace pbs
