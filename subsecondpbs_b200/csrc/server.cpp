// Dose-request server (see server.h) and its C ABI (include/subsecondpbs.h).
#include "server.h"

#include <algorithm>
#include <cstring>
#include <new>
#include <system_error>

#include "kernels.h"
#include "plan.h"

namespace pbs {

namespace {

template <class T>
const T* copy_array(std::vector<T>& dst, const T* src, size_t n) {
    if (!src || n == 0) {
        dst.clear();
        return nullptr;
    }
    dst.assign(src, src + n);
    return dst.data();
}

int fail(int rc, const std::string& msg) {
    set_error(msg);
    return rc;
}

size_t grid_voxels(const GridDesc& g) { return size_t(g.dims[0]) * size_t(g.dims[1]) * size_t(g.dims[2]); }

bool grid_ok(const GridDesc& g) {
    return g.dims[0] > 0 && g.dims[1] > 0 && g.dims[2] > 0 && g.res[0] > 0.0f && g.res[1] > 0.0f && g.res[2] > 0.0f;
}

constexpr size_t kMaxPooledResults = 64;

}  // namespace

void OwnedBeam::assign(const PbsBeamDesc& b) {
    d = b;
    d.energies = copy_array(energies, b.energies, b.n_energies);
    d.spot_sigmas = copy_array(sigmas, b.spot_sigmas, b.n_spot_sigmas);
    d.subspot_data = copy_array(subspots, b.subspot_data, b.n_subspot_data);
    d.layer_spot_counts = copy_array(counts, b.layer_spot_counts, b.n_layer_spot_counts);
    d.spot_positions = copy_array(positions, b.spot_positions, b.n_spot_positions);
    d.spot_weights = copy_array(weights, b.spot_weights, b.n_spot_weights);
    d.spot_beam_directions = copy_array(directions, b.spot_beam_directions, b.n_spot_beam_directions);
    d.layer_longitudinal_cutoffs = copy_array(cutoffs, b.layer_longitudinal_cutoffs, b.n_layer_longitudinal_cutoffs);
    d.water_equivalence = copy_array(weq, b.water_equivalence, b.n_water_equivalence);
    d.ray_weq_header = copy_array(weqHeader, b.ray_weq_header, b.n_ray_weq_header);
    d.profile_data = copy_array(profile, b.profile_data, b.n_profile_data);
    d.profile_setting = copy_array(profileSetting, b.profile_setting, b.n_profile_setting);
    d.beam_para_data = copy_array(beamPara, b.beam_para_data, b.n_beam_para_data);
    d.roi_linear_indices = copy_array(roi, b.roi_linear_indices, b.n_roi_linear_indices);
}

void OwnedEnergy::assign(const PbsEnergyDesc& e) {
    d = e;
    d.energies_per_u = copy_array(energiesPerU, e.energies_per_u, e.n_energies_per_u);
    d.peak_depths = copy_array(peakDepths, e.peak_depths, e.n_peak_depths);
    d.scale_facts = copy_array(scaleFacts, e.scale_facts, e.n_scale_facts);
    d.cidd_matrix = copy_array(cidd, e.cidd_matrix, e.n_cidd_matrix);
    d.density_vector = copy_array(density, e.density_vector, e.n_density_vector);
    d.sp_vector = copy_array(sp, e.sp_vector, e.n_sp_vector);
    d.rrl_vector = copy_array(rrl, e.rrl_vector, e.n_rrl_vector);
    d.nuc_weight_matrix = copy_array(nucWeight, e.nuc_weight_matrix, e.n_nuc_weight_matrix);
    d.nuc_sq_sigma_matrix = copy_array(nucSqSigma, e.nuc_sq_sigma_matrix, e.n_nuc_sq_sigma_matrix);
    // FNV-1a over everything the tracer reads from the tables.
    unsigned long long h = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    };
    mix(density.data(), density.size() * 4);
    mix(sp.data(), sp.size() * 4);
    mix(&e.n_density_samples, sizeof(int));
    mix(&e.n_sp_samples, sizeof(int));
    mix(&e.density_scale_fact, sizeof(float));
    mix(&e.sp_scale_fact, sizeof(float));
    lutHash = h;
}

namespace {
// Identity of a trace within one patient: the tracer geometry, the ray grid, the
// step count and the tracer's tables.
std::string trace_key(const TracerParams& t, int rayX, int rayY, int steps, unsigned long long lutHash) {
    std::string k(reinterpret_cast<const char*>(&t), sizeof(TracerParams));
    const int v[3] = {rayX, rayY, steps};
    k.append(reinterpret_cast<const char*>(v), sizeof(v));
    k.append(reinterpret_cast<const char*>(&lutHash), sizeof(lutHash));
    return k;
}
}  // namespace

int SlotTraces::acquire(Context&, const BeamGeomDev& g, TraceSlot& ts) { return server->trace_acquire(*slot, g, ts); }

int SlotTraces::traced(Context&, TraceSlot& ts) { return server->trace_done(*slot, ts); }

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stopping_ = true;
    }
    cvWork_.notify_all();
    for (auto& s : slots_)
        if (s->thread.joinable()) s->thread.join();
    cudaSetDevice(device_);
    cudaStream_t st = slots_.empty() ? nullptr : slots_.front()->ctx.stream;
    for (auto& kv : patients_) {
        Patient& p = *kv.second;
        if (p.deviceCt) cudaFreeAsync(p.deviceCt, st);
        p.hostCt.release();
        if (p.ready) cudaEventDestroy(p.ready);
        for (auto& tv : p.traces) {
            if (tv.second->mem) cudaFreeAsync(tv.second->mem, st);
            if (tv.second->ready) cudaEventDestroy(tv.second->ready);
        }
    }
    if (st) cudaStreamSynchronize(st);
    for (auto& kv : requests_) kv.second->result.release();
    for (auto& kv : freeResults_) cudaFreeHost(kv.second);
    slots_.clear();
}

double Server::now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

int Server::init(int gpu, int nSlots, size_t budgetBytes) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || gpu < 0 || gpu >= n)
        return fail(PBS_ERR_INVALID_ARGUMENT, "gpu_id " + std::to_string(gpu) + " out of range");
    if (nSlots < 1 || nSlots > 64) return fail(PBS_ERR_INVALID_ARGUMENT, "a server needs 1 to 64 slots");
    device_ = gpu;
    if (cudaSetDevice(gpu) != cudaSuccess) return fail(PBS_ERR_CUDA, "cudaSetDevice failed");
    if (budgetBytes == 0) {
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return fail(PBS_ERR_CUDA, "cudaMemGetInfo failed");
        budgetBytes = freeB / 10 * 9;
    }
    budget_ = budgetBytes;
    t0_ = std::chrono::steady_clock::now();
    for (int i = 0; i < nSlots; ++i) {
        auto s = std::make_unique<Slot>();
        s->index = i;
        int rc = s->ctx.init(gpu);
        if (rc) return rc;
        s->ctx.use_stream_ordered_allocation();
        // Pinned staging for the beams' host inputs, sized up front for the same reason
        // as the result buffers (see add_patient); larger beams still grow it.
        if ((rc = s->ctx.staging.ensure(size_t(4) << 20))) return rc;
        s->traces.server = this;
        s->traces.slot = s.get();
        s->ctx.traceStore = &s->traces;
        s->ctx.layerBudgetMiB = layerBudgetMiB_;
        s->ctx.nuclearModel = nuclearModel_;
        s->bytes = s->ctx.device_bytes();
        slots_.push_back(std::move(s));
    }
    for (auto& s : slots_) s->thread = std::thread(&Server::worker, this, s.get());
    return PBS_OK;
}

int Server::set_option(int option, long long value) {
    std::lock_guard<std::mutex> lk(mu_);
    if (running_ > 0 || !queue_.empty()) return fail(PBS_ERR_NOT_READY, "server options change only while it is idle");
    for (auto& s : slots_) {
        Context& c = s->ctx;
        switch (option) {
            case PBS_OPT_COMPAT_BEV_Z_SHIFT: c.compatBevZShift = value != 0; break;
            case PBS_OPT_LAYER_BUDGET_MIB: c.layerBudgetMiB = value; break;
            case PBS_OPT_NUCLEAR_MODEL:
                if (value < 0 || value > 2) return fail(PBS_ERR_INVALID_ARGUMENT, "nuclear model must be 0, 1 or 2");
                c.nuclearModel = int(value);
                break;
            default: return fail(PBS_ERR_UNSUPPORTED, "option not available on a server");
        }
    }
    if (option == PBS_OPT_LAYER_BUDGET_MIB) layerBudgetMiB_ = value;
    if (option == PBS_OPT_NUCLEAR_MODEL) nuclearModel_ = int(value);
    if (option == PBS_OPT_COMPAT_BEV_Z_SHIFT) compatBevZShift_ = value != 0;
    return PBS_OK;
}

int Server::set_trace_cache(bool on) {
    std::lock_guard<std::mutex> lk(mu_);
    if (running_ > 0 || !queue_.empty()) return fail(PBS_ERR_NOT_READY, "server options change only while it is idle");
    traceCache = on;
    return PBS_OK;
}

int Server::add_energy(int id, const PbsEnergyDesc& e) {
    if (!(e.n_energies > 0 && e.n_energy_samples > 0) || !e.energies_per_u || !e.cidd_matrix ||
        e.n_cidd_matrix != size_t(e.n_energies) * size_t(e.n_energy_samples))
        return fail(PBS_ERR_INVALID_ARGUMENT, "[RTD_ENTRY_ASSERT] energy table dimensions are inconsistent");
    auto owned = std::make_unique<OwnedEnergy>();
    owned->assign(e);
    std::lock_guard<std::mutex> lk(mu_);
    if (energies_.count(id)) return fail(PBS_ERR_INVALID_ARGUMENT, "energy id " + std::to_string(id) + " exists");
    energies_[id] = std::move(owned);
    return PBS_OK;
}

int Server::add_patient(int id, const float* ct, const GridDesc& ctGrid, const GridDesc& doseGrid) {
    if (!ct || !grid_ok(ctGrid) || !grid_ok(doseGrid))
        return fail(PBS_ERR_INVALID_ARGUMENT, "[RTD_ENTRY_ASSERT] CT and dose grids need positive dims and resolution");
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (patients_.count(id)) return fail(PBS_ERR_INVALID_ARGUMENT, "patient id " + std::to_string(id) + " exists");
    }
    if (cudaSetDevice(device_) != cudaSuccess) return fail(PBS_ERR_CUDA, "cudaSetDevice failed");
    auto p = std::make_unique<Patient>();
    p->id = id;
    p->ctGrid = ctGrid;
    p->doseGrid = doseGrid;
    const size_t n = grid_voxels(ctGrid);
    p->ctBytes = n * 4;
    int rc = p->hostCt.ensure(p->ctBytes);
    if (rc) return rc;
    std::memcpy(p->hostCt.ptr, ct, p->ctBytes);
    int type = parse_ct_input_type_env();
    if (type == PBS_CT_AUTO) {
        float mn, mx;
        sample_ct_stats(ct, n, mn, mx);
        type = auto_detect_ct_type(mn, mx);
    }
    p->ctType = type;
    if (cudaEventCreateWithFlags(&p->ready, cudaEventDisableTiming) != cudaSuccess) {
        p->hostCt.release();
        return fail(PBS_ERR_CUDA, "cudaEventCreate failed");
    }
    const size_t resultBytes = grid_voxels(doseGrid) * 4;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (patients_.count(id)) {
            p->hostCt.release();
            cudaEventDestroy(p->ready);
            return fail(PBS_ERR_INVALID_ARGUMENT, "patient id " + std::to_string(id) + " exists");
        }
        patients_[id] = std::move(p);
    }
    // Pinned result buffers of this grid size for every slot and two in the
    // caller's hands, allocated now: pinning host memory while requests run
    // stalls the device.
    const size_t want = slots_.size() + 2;
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(poolMu_);
            if (freeResults_.count(resultBytes) >= want || freeResults_.size() >= kMaxPooledResults) break;
        }
        void* ptr = nullptr;
        if (cudaMallocHost(&ptr, resultBytes) != cudaSuccess) break;  // the pool grows on demand instead
        std::lock_guard<std::mutex> lk(poolMu_);
        freeResults_.emplace(resultBytes, ptr);
    }
    return PBS_OK;
}

int Server::remove_patient(int id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = patients_.find(id);
    if (it == patients_.end()) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown patient " + std::to_string(id));
    Patient& p = *it->second;
    bool queued = false;
    for (const Request* r : queue_) queued = queued || r->patient == &p;
    if (p.pins > 0 || queued || p.state == Patient::Loading)
        return fail(PBS_ERR_NOT_READY, "patient " + std::to_string(id) + " has requests queued or running");
    cudaSetDevice(device_);
    cudaStream_t st = slots_.front()->ctx.stream;
    if (p.deviceCt) {
        // No request uses the CT any more (every user's stream was synchronised).
        cudaFreeAsync(p.deviceCt, st);
        residentBytes_ -= p.ctBytes;
    }
    for (auto& tv : p.traces) {
        if (tv.second->mem) evict_trace(*tv.second, st);
        if (tv.second->ready) cudaEventDestroy(tv.second->ready);
    }
    p.hostCt.release();
    cudaEventDestroy(p.ready);
    patients_.erase(it);
    return PBS_OK;
}

int Server::submit(int patientId, int energyId, const PbsBeamDesc* beams, size_t nBeams, int nuclear,
                   unsigned long long* ticket) {
    if (!beams || nBeams == 0 || !ticket) return fail(PBS_ERR_INVALID_ARGUMENT, "submit needs beams and a ticket");
    Patient* p = nullptr;
    OwnedEnergy* e = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto pi = patients_.find(patientId);
        auto ei = energies_.find(energyId);
        if (pi == patients_.end()) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown patient " + std::to_string(patientId));
        if (ei == energies_.end()) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown energy id " + std::to_string(energyId));
        p = pi->second.get();
        e = ei->second.get();
    }
    auto r = std::make_unique<Request>();
    r->patientId = patientId;
    r->energyId = energyId;
    r->nuclear = nuclear != 0;
    r->patient = p;
    r->energy = e;
    r->beams.resize(nBeams);
    // Device bytes of the request on a slot: tables, FP64 grid and its float copy,
    // and the largest beam's working set (the beams run one after another).
    size_t maxBeam = 0;
    for (size_t i = 0; i < nBeams; ++i) {
        r->beams[i].assign(beams[i]);
        std::string err;
        if (!validate_beam(r->beams[i].d, 0, err)) return fail(PBS_ERR_INVALID_ARGUMENT, err);
        BeamPlan plan;
        int rc = plan_beam(r->beams[i].d, e->d, p->ctGrid, p->doseGrid, plan, err);
        if (rc) return fail(rc, err);
        const BeamBuffers z = beam_buffers(plan, r->beams[i].d.n_subspot_data, r->nuclear, layerBudgetMiB_);
        maxBeam = std::max(maxBeam, z.total(!traceCache));
        if (traceCache && !plan.hasWeqVolume) {
            r->traceKeys.push_back(trace_key(plan.tracer, plan.rayDims[0], plan.rayDims[1], plan.tracerSteps, e->lutHash));
            r->traceBytes.push_back(trace_bytes(size_t(plan.tracerSteps), size_t(plan.rayDims[0]) * plan.rayDims[1]));
        }
    }
    const size_t tableBytes = (e->cidd.size() + e->density.size() + e->sp.size() + e->rrl.size() +
                               e->nucWeight.size() + e->nucSqSigma.size()) * 4;
    r->estBytes = maxBeam + grid_voxels(p->doseGrid) * 12 + tableBytes + 4096;
    size_t traceTotal = 0;
    for (size_t b : r->traceBytes) traceTotal += b;
    if (r->estBytes + p->ctBytes + traceTotal > budget_)
        return fail(PBS_ERR_OUT_OF_MEMORY, "request needs " + std::to_string((r->estBytes + p->ctBytes + traceTotal) >> 20) +
                                               " MiB of device memory; the server budget is " +
                                               std::to_string(budget_ >> 20) + " MiB");
    std::lock_guard<std::mutex> lk(mu_);
    if (stopping_) return fail(PBS_ERR_NOT_READY, "server is stopping");
    r->ticket = nextTicket_++;
    r->tSubmit = now();
    *ticket = r->ticket;
    queue_.push_back(r.get());
    requests_[r->ticket] = std::move(r);
    ++submitted_;
    cvWork_.notify_all();
    return PBS_OK;
}

size_t Server::committed_bytes() const {
    size_t n = residentBytes_;
    for (const auto& s : slots_) n += s->current ? std::max(s->bytes, s->current->estBytes) : s->bytes;
    return n;
}

void Server::evict_trace(TraceEntry& e, cudaStream_t st) {
    // Every request that read the trace has completed and synchronised its stream.
    cudaFreeAsync(e.mem, st);
    e.mem = nullptr;
    e.slot = TraceSlot{};
    e.state = TraceEntry::Absent;
    residentBytes_ -= e.bytes;
}

bool Server::make_room(size_t need, const Request& r, Slot& self) {
    size_t committed = committed_bytes();
    const Patient* keep = r.patient;
    auto wanted = [&](const Patient& p, const std::string& key) {
        if (&p != keep) return false;
        for (const std::string& k : r.traceKeys)
            if (k == key) return true;
        return false;
    };
    while (committed + need > budget_) {
        // Least recently used idle CT or trace.
        Patient* vp = nullptr;
        TraceEntry* vt = nullptr;
        unsigned long long oldest = ~0ull;
        for (auto& kv : patients_) {
            Patient* q = kv.second.get();
            if (q != keep && q->state == Patient::Resident && q->pins == 0 && q->lastUse < oldest) {
                oldest = q->lastUse;
                vp = q;
                vt = nullptr;
            }
            for (auto& tv : q->traces) {
                TraceEntry* e = tv.second.get();
                if (e->state == TraceEntry::Ready && e->pins == 0 && e->lastUse < oldest && !wanted(*q, tv.first)) {
                    oldest = e->lastUse;
                    vt = e;
                    vp = nullptr;
                }
            }
        }
        if (vt) {
            committed -= vt->bytes;
            evict_trace(*vt, self.ctx.stream);
            ++traceEvictions_;
            continue;
        }
        if (!vp) break;
        // Every request that read the CT has completed and synchronised its stream.
        cudaFreeAsync(vp->deviceCt, self.ctx.stream);
        vp->deviceCt = nullptr;
        vp->state = Patient::Absent;
        residentBytes_ -= vp->ctBytes;
        committed -= vp->ctBytes;
        ++evictions_;
    }
    for (auto& o : slots_) {
        if (committed + need <= budget_) break;
        if (o.get() == &self || o->current || o->bytes == 0) continue;
        // An idle slot's stream has no work left; its thread is waiting for the lock.
        const size_t before = o->bytes;
        o->ctx.release_beam_buffers();
        o->bytes = o->ctx.device_bytes();
        committed -= before - o->bytes;
        ++slotReleases_;
    }
    return committed + need <= budget_;
}

Request* Server::pick(Slot& s) {
    if (queue_.empty()) return nullptr;
    const double t = now();
    const bool headBlocks = t - queue_.front()->tSubmit > maxBypassSec;
    for (size_t i = 0; i < queue_.size(); ++i) {
        if (i > 0 && headBlocks) break;
        Request* r = queue_[i];
        Patient* p = r->patient;
        size_t traceNeed = 0;
        for (size_t k = 0; k < r->traceKeys.size(); ++k) {
            bool dup = false;
            for (size_t j = 0; j < k; ++j) dup = dup || r->traceKeys[j] == r->traceKeys[k];
            auto it = p->traces.find(r->traceKeys[k]);
            if (!dup && (it == p->traces.end() || it->second->state == TraceEntry::Absent)) traceNeed += r->traceBytes[k];
        }
        const size_t need = (r->estBytes > s.bytes ? r->estBytes - s.bytes : 0) +
                            (p->state == Patient::Absent ? p->ctBytes : 0) + traceNeed;
        if (committed_bytes() + need > budget_ && !make_room(need, *r, s)) continue;
        queue_.erase(queue_.begin() + long(i));
        r->slot = s.index;
        r->state = 1;
        r->tStart = t;
        r->loadsPatient = p->state == Patient::Absent;
        if (r->loadsPatient) {
            p->state = Patient::Loading;
            residentBytes_ += p->ctBytes;
        }
        ++p->pins;
        p->lastUse = ++useClock_;
        r->traces.assign(r->traceKeys.size(), nullptr);
        for (size_t k = 0; k < r->traceKeys.size(); ++k) {
            std::unique_ptr<TraceEntry>& e = p->traces[r->traceKeys[k]];
            if (!e) {
                e = std::make_unique<TraceEntry>();
                e->bytes = r->traceBytes[k];
                cudaEventCreateWithFlags(&e->ready, cudaEventDisableTiming);
            }
            if (e->state == TraceEntry::Absent) {
                e->state = TraceEntry::Loading;
                e->loader = r;
                residentBytes_ += e->bytes;
            }
            ++e->pins;
            e->lastUse = ++useClock_;
            r->traces[k] = e.get();
        }
        s.current = r;
        ++running_;
        peakBytes_ = std::max(peakBytes_, committed_bytes());
        return r;
    }
    return nullptr;
}

void Server::worker(Slot* s) {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        Request* r = nullptr;
        while (!stopping_ && !(r = pick(*s))) cvWork_.wait(lk);
        if (!r) break;
        lk.unlock();
        const int rc = execute(*s, *r);
        const std::string err = rc ? std::string(last_error()) : std::string();
        lk.lock();
        r->rc = rc;
        r->error = err;
        r->tDone = now();
        r->state = 2;
        --r->patient->pins;
        for (TraceEntry* e : r->traces) {
            if (!e) continue;
            --e->pins;
            if (e->loader == r) {
                e->loader = nullptr;
                if (e->state == TraceEntry::Loading) {  // the request failed before tracing
                    if (e->mem) cudaFreeAsync(e->mem, s->ctx.stream);
                    e->mem = nullptr;
                    e->slot = TraceSlot{};
                    e->state = TraceEntry::Absent;
                    residentBytes_ -= e->bytes;
                    cvLoad_.notify_all();
                }
            }
        }
        s->current = nullptr;
        s->bytes = s->ctx.device_bytes();
        --running_;
        if (rc)
            ++failed_;
        else
            ++completed_;
        cvDone_.notify_all();
        cvWork_.notify_all();
    }
}

int Server::trace_acquire(Slot& s, const BeamGeomDev& g, TraceSlot& ts) {
    Request* r = s.current;
    if (!traceCache || !r) return PBS_OK;
    const std::string key = trace_key(g.tracer, g.rayX, g.rayY, g.steps, r->energy->lutHash);
    TraceEntry* e = nullptr;
    for (size_t k = 0; k < r->traceKeys.size() && !e; ++k)
        if (r->traceKeys[k] == key) e = r->traces[k];
    if (!e) return PBS_OK;  // not planned at submit: the context traces into its own buffers
    std::unique_lock<std::mutex> lk(mu_);
    if (e->state == TraceEntry::Loading && e->loader == r && !e->mem) {
        lk.unlock();
        const size_t rays = size_t(g.rayX) * g.rayY, S = size_t(g.steps);
        void* mem = nullptr;
        cudaError_t err = cudaMallocAsync(&mem, e->bytes, s.ctx.stream);
        if (err != cudaSuccess)
            return fail(err == cudaErrorMemoryAllocation ? PBS_ERR_OUT_OF_MEMORY : PBS_ERR_CUDA,
                        std::string("trace allocation: ") + cudaGetErrorString(err));
        auto up = [](size_t n) { return (n + 255) / 256 * 256; };
        char* p = static_cast<char*>(mem);
        TraceSlot t;
        t.dens = reinterpret_cast<float*>(p);
        p += up(S * rays * 4);
        t.wepl = reinterpret_cast<float*>(p);
        p += up(S * rays * 4);
        t.firstIn = reinterpret_cast<int*>(p);
        p += up(rays * 4);
        t.firstOut = reinterpret_cast<int*>(p);
        p += up(rays * 4);
        t.weplMin = reinterpret_cast<float*>(p);
        p += up(S * 4);
        t.inOut = reinterpret_cast<int*>(p);
        lk.lock();
        e->mem = mem;
        e->slot = t;
        ++traceLoads_;
        ts = t;
        ts.traced = false;
        return PBS_OK;
    }
    if (!cvLoad_.wait_for(lk, std::chrono::seconds(120), [&] { return e->state != TraceEntry::Loading; }))
        return fail(PBS_ERR_TIMEOUT, "timed out waiting for a resident trace");
    if (e->state != TraceEntry::Ready) return fail(PBS_ERR_CUDA, "a resident trace failed to build");
    ts = e->slot;
    ts.traced = true;
    ts.ready = e->ready;
    ++traceHits_;
    return PBS_OK;
}

int Server::trace_done(Slot& s, TraceSlot& ts) {
    Request* r = s.current;
    TraceEntry* e = nullptr;
    for (TraceEntry* q : r->traces)
        if (q && q->slot.dens == ts.dens) e = q;
    if (!e) return fail(PBS_ERR_CUDA, "trace_done: unknown trace");
    if (cudaEventRecord(e->ready, s.ctx.stream) != cudaSuccess) return fail(PBS_ERR_CUDA, "cudaEventRecord failed");
    std::lock_guard<std::mutex> lk(mu_);
    e->state = TraceEntry::Ready;
    cvLoad_.notify_all();
    return PBS_OK;
}

int Server::ensure_resident(Slot& s, Request& r) {
    Patient& p = *r.patient;
    Context& c = s.ctx;
    if (r.loadsPatient) {
        int rc = PBS_OK;
        cudaError_t e = cudaMallocAsync(&p.deviceCt, p.ctBytes, c.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(p.deviceCt, p.hostCt.ptr, p.ctBytes, cudaMemcpyHostToDevice, c.stream);
        if (e != cudaSuccess) {
            rc = e == cudaErrorMemoryAllocation ? PBS_ERR_OUT_OF_MEMORY : PBS_ERR_CUDA;
            set_error(std::string("patient CT upload: ") + cudaGetErrorString(e));
        }
        if (!rc) rc = c.convert_ct_buffer(static_cast<float*>(p.deviceCt), p.ctBytes / 4, p.ctType);
        if (!rc && cudaEventRecord(p.ready, c.stream) != cudaSuccess) rc = fail(PBS_ERR_CUDA, "cudaEventRecord failed");
        std::lock_guard<std::mutex> lk(mu_);
        if (rc) {
            if (p.deviceCt) cudaFreeAsync(p.deviceCt, c.stream);
            p.deviceCt = nullptr;
            p.state = Patient::Absent;
            residentBytes_ -= p.ctBytes;
        } else {
            p.state = Patient::Resident;
            ++p.loads;
            ++loads_;
        }
        cvLoad_.notify_all();
        return rc;
    }
    cudaEvent_t ready = nullptr;
    {
        std::unique_lock<std::mutex> lk(mu_);
        // The loader only enqueues the upload before it flips the state, so this
        // wait is short; it is bounded all the same.
        if (!cvLoad_.wait_for(lk, std::chrono::seconds(120), [&] { return p.state != Patient::Loading; }))
            return fail(PBS_ERR_TIMEOUT, "timed out waiting for patient " + std::to_string(p.id) + " to load");
        if (p.state != Patient::Resident)
            return fail(PBS_ERR_CUDA, "patient " + std::to_string(p.id) + " failed to load");
        ready = p.ready;
    }
    if (cudaStreamWaitEvent(c.stream, ready, 0) != cudaSuccess) return fail(PBS_ERR_CUDA, "cudaStreamWaitEvent failed");
    return PBS_OK;
}

int Server::acquire_result(Request& r, size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(poolMu_);
        auto it = freeResults_.find(bytes);
        if (it != freeResults_.end()) {
            r.result.ptr = it->second;
            r.result.bytes = bytes;
            freeResults_.erase(it);
            return PBS_OK;
        }
    }
    return r.result.ensure(bytes);
}

void Server::recycle_result(PinnedBuf& b) {
    if (!b.ptr) return;
    {
        std::lock_guard<std::mutex> lk(poolMu_);
        if (freeResults_.size() < kMaxPooledResults) {
            freeResults_.emplace(b.bytes, b.ptr);
            b.ptr = nullptr;
            b.bytes = 0;
            return;
        }
    }
    b.release();
}

int Server::execute(Slot& s, Request& r) {
    Context& c = s.ctx;
    if (cudaSetDevice(device_) != cudaSuccess) return fail(PBS_ERR_CUDA, "cudaSetDevice failed");
    const OwnedEnergy* e = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu_);
        e = energies_.at(r.energyId).get();
    }
    const Patient& p = *r.patient;
    int rc = c.set_energy(e->d);
    if (!rc) rc = ensure_resident(s, r);
    if (!rc) rc = c.attach_ct(static_cast<const float*>(p.deviceCt), p.ctGrid, p.ctType);
    if (!rc) rc = c.set_dose_grid(p.doseGrid);
    for (size_t i = 0; !rc && i < r.beams.size(); ++i) rc = c.add_beam(r.beams[i].d, r.nuclear);
    if (!rc) rc = acquire_result(r, grid_voxels(p.doseGrid) * 4);
    r.tEnqueued = now();
    if (!rc) rc = c.read_dose(static_cast<float*>(r.result.ptr), 0);
    if (rc) {
        // Leave the slot idle and clean for the next request.
        const std::string msg = last_error();
        cudaStreamSynchronize(c.stream);
        c.take_device_errors();
        set_error(msg);
    }
    c.ctView = nullptr;
    c.hasCt = false;
    return rc;
}

int Server::wait(unsigned long long ticket, double timeoutSec, const float** dose, double times[3], int* slot) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = requests_.find(ticket);
    if (it == requests_.end()) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown ticket " + std::to_string(ticket));
    Request* r = it->second.get();
    auto done = [&] { return r->state == 2; };
    if (timeoutSec < 0.0)
        cvDone_.wait(lk, done);
    else if (!cvDone_.wait_for(lk, std::chrono::duration<double>(timeoutSec), done))
        return fail(PBS_ERR_TIMEOUT, "request " + std::to_string(ticket) + " not finished");
    if (times) {
        times[0] = r->tSubmit;
        times[1] = r->tStart;
        times[2] = r->tDone;
    }
    if (slot) *slot = r->slot;
    if (r->rc) return fail(r->rc, r->error);
    if (dose) *dose = static_cast<const float*>(r->result.ptr);
    return PBS_OK;
}

int Server::info(unsigned long long ticket, double times[4], int* slot, long long* estBytes) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = requests_.find(ticket);
    if (it == requests_.end()) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown ticket " + std::to_string(ticket));
    const Request& r = *it->second;
    if (r.state != 2) return fail(PBS_ERR_NOT_READY, "request is still queued or running");
    if (times) {
        times[0] = r.tSubmit;
        times[1] = r.tStart;
        times[2] = r.tEnqueued;
        times[3] = r.tDone;
    }
    if (slot) *slot = r.slot;
    if (estBytes) *estBytes = static_cast<long long>(r.estBytes);
    return PBS_OK;
}

int Server::release(unsigned long long ticket) {
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = requests_.find(ticket);
        if (it == requests_.end()) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown ticket " + std::to_string(ticket));
        if (it->second->state != 2) return fail(PBS_ERR_NOT_READY, "request is still queued or running");
        r = std::move(it->second);
        requests_.erase(it);
    }
    recycle_result(r->result);
    return PBS_OK;
}

int Server::drain(double timeoutSec) {
    std::unique_lock<std::mutex> lk(mu_);
    auto idle = [&] { return queue_.empty() && running_ == 0; };
    if (timeoutSec < 0.0) {
        cvDone_.wait(lk, idle);
        return PBS_OK;
    }
    if (!cvDone_.wait_for(lk, std::chrono::duration<double>(timeoutSec), idle))
        return fail(PBS_ERR_TIMEOUT, "server did not drain in time");
    return PBS_OK;
}

void Server::stats(ServerStats* out) {
    std::lock_guard<std::mutex> lk(mu_);
    out->submitted = submitted_;
    out->completed = completed_;
    out->failed = failed_;
    out->queued = static_cast<long long>(queue_.size());
    out->running = running_;
    out->patientLoads = loads_;
    out->evictions = evictions_;
    out->slotReleases = slotReleases_;
    out->traceHits = traceHits_;
    out->traceLoads = traceLoads_;
    out->traceEvictions = traceEvictions_;
    out->residentBytes = residentBytes_;
    size_t sb = 0;
    for (const auto& s : slots_) sb += s->bytes;
    out->slotBytes = sb;
    out->peakBytes = peakBytes_;
    out->budgetBytes = budget_;
}

}  // namespace pbs

// ---- C ABI ------------------------------------------------------------------

struct PbsServer {
    pbs::Server server;
};

namespace {

pbs::GridDesc make_grid(const int dims[3], const float res[3], const float corner[3]) {
    pbs::GridDesc g{};
    for (int i = 0; i < 3; ++i) {
        g.dims[i] = dims[i];
        g.res[i] = res[i];
        g.corner[i] = corner[i];
    }
    return g;
}

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        pbs::set_error("host allocation failed");
        return PBS_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& ex) {
        pbs::set_error(ex.what());
        return PBS_ERR_CUDA;
    }
}

}  // namespace

extern "C" {

PBS_API int pbs_server_create(int gpu_id, int n_slots, long long hbm_budget_mib, PbsServer** out) {
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    return guarded([&] {
        auto s = std::make_unique<PbsServer>();
        const size_t budget = hbm_budget_mib > 0 ? size_t(hbm_budget_mib) << 20 : 0;
        int rc = s->server.init(gpu_id, n_slots, budget);
        if (rc) return rc;
        *out = s.release();
        return int(PBS_OK);
    });
}

PBS_API int pbs_server_destroy(PbsServer* s) {
    delete s;
    return PBS_OK;
}

PBS_API int pbs_server_set_option(PbsServer* s, int option, long long value) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.set_option(option, value); });
}

PBS_API int pbs_server_set_bypass_limit(PbsServer* s, double seconds) {
    if (!s || !(seconds >= 0.0)) return PBS_ERR_INVALID_ARGUMENT;
    s->server.maxBypassSec = seconds;
    return PBS_OK;
}

PBS_API int pbs_server_set_trace_cache(PbsServer* s, int enabled) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.set_trace_cache(enabled != 0); });
}

PBS_API int pbs_server_add_energy(PbsServer* s, int energy_id, const PbsEnergyDesc* energy) {
    if (!s || !energy) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.add_energy(energy_id, *energy); });
}

PBS_API int pbs_server_add_patient(PbsServer* s, int patient_id, const float* ct, const int ct_dims[3],
                                   const float ct_resolution[3], const float ct_corner[3], const int dose_dims[3],
                                   const float dose_resolution[3], const float dose_corner[3]) {
    if (!s || !ct_dims || !ct_resolution || !ct_corner || !dose_dims || !dose_resolution || !dose_corner)
        return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] {
        return s->server.add_patient(patient_id, ct, make_grid(ct_dims, ct_resolution, ct_corner),
                                     make_grid(dose_dims, dose_resolution, dose_corner));
    });
}

PBS_API int pbs_server_remove_patient(PbsServer* s, int patient_id) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.remove_patient(patient_id); });
}

PBS_API int pbs_server_submit(PbsServer* s, int patient_id, int energy_id, const PbsBeamDesc* beams, size_t n_beams,
                              int nuclear_correction, unsigned long long* ticket) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.submit(patient_id, energy_id, beams, n_beams, nuclear_correction, ticket); });
}

PBS_API int pbs_server_wait(PbsServer* s, unsigned long long ticket, double timeout_s, const float** dose,
                            double times[3], int* slot) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.wait(ticket, timeout_s, dose, times, slot); });
}

PBS_API int pbs_server_request_info(PbsServer* s, unsigned long long ticket, double times[4], int* slot,
                                    long long* est_bytes) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.info(ticket, times, slot, est_bytes); });
}

PBS_API int pbs_server_release(PbsServer* s, unsigned long long ticket) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.release(ticket); });
}

PBS_API int pbs_server_drain(PbsServer* s, double timeout_s) {
    if (!s) return PBS_ERR_INVALID_ARGUMENT;
    return guarded([&] { return s->server.drain(timeout_s); });
}

PBS_API int pbs_server_stats(PbsServer* s, PbsServerStats* out) {
    if (!s || !out) return PBS_ERR_INVALID_ARGUMENT;
    pbs::ServerStats st;
    s->server.stats(&st);
    out->submitted = st.submitted;
    out->completed = st.completed;
    out->failed = st.failed;
    out->queued = st.queued;
    out->running = st.running;
    out->patient_loads = st.patientLoads;
    out->evictions = st.evictions;
    out->slot_releases = st.slotReleases;
    out->resident_bytes = (long long)st.residentBytes;
    out->slot_bytes = (long long)st.slotBytes;
    out->peak_bytes = (long long)st.peakBytes;
    out->budget_bytes = (long long)st.budgetBytes;
    out->trace_hits = st.traceHits;
    out->trace_loads = st.traceLoads;
    out->trace_evictions = st.traceEvictions;
    return PBS_OK;
}

PBS_API double pbs_server_now(PbsServer* s) { return s ? s->server.now() : 0.0; }

}  // extern "C"
