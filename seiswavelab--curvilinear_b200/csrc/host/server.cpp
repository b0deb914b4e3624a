// Serving request loop (include/swl_server.h): admission by device-memory budget, model builds
// on a host thread pool, and scheduler threads that keep a batch in flight on every running
// shot.  Each shot owns its engine and CUDA stream, so batches of different shots overlap on
// the GPU.  In the persistent form the 2D shots instead advance together: one host thread
// gathers the running 2D shots of each (precision, GSLS mechanism count) into one persistent
// multi-shot launch per round, admits new shots at the next round, and records each shot's batch
// when the launch completes.  Finished shots release their device memory at once, which admits
// the next request.
#include "../../../include/swl_fleet.h"
#include "../../../include/swl_server.h"
#include "sessions.hpp"
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

namespace swl::host {

struct Shot {
    int64_t id{};
    int dim{2};
    int state{SWL_SHOT_QUEUED};
    Params2D p2;
    Params3D p3;
    std::unique_ptr<Session2D> s2;
    std::unique_ptr<Session3D> s3;
    double submit{}, start{}, finish{}, run{};
    std::string error;
    int64_t bytes{}; // device bytes charged against the budget
    int steps() const { return dim == 2 ? (s2 ? s2->step : 0) : (s3 ? s3->step : 0); }
    int total() const { return dim == 2 ? (s2 ? s2->model.total : 0) : (s3 ? s3->model.total : 0); }
};

// Device bytes of a request before its model exists (src/two_d/MemoryBudget2D.hpp:12-38 style), an
// upper bound of what its engine will hold: the state sets (six in FP32, with the compensation),
// the model arrays, the ADE memories, the trace table of the largest batch, and an allowance.
int64_t estimate(const Shot &s) {
    constexpr double allowance = double(64ll << 20);
    if (s.dim == 2) {
        const auto &p = s.p2;
        const int wx = std::clamp(p.spongeX, 1, std::max(1, p.nx / 3)), wz = std::clamp(p.spongeZ, 1, std::max(1, p.nz / 3));
        const bool ext = p.absorbing && p.externalAbsorption;
        const int nxp = p.nx + 6 + (ext ? 2 * wx : 0), nzp = p.nz + 6 + (ext ? wz : 0);
        const double n = double((nxp + 1 + 7) / 8 * 8) * nzp; // pitched rows
        const int L = p.attenuation.enabled ? p.attenuation.mechanisms : 0, fc = L ? 6 + 4 * L : 5;
        const double b = p.precision == SWL_FP32 ? 4 : 8, sets = p.precision == SWL_FP32 ? 6 : 4;
        const double cpml = p.absorbing && p.absorber == 1 ? 4.0 * (2.0 * wx * nzp + double(wz) * nxp) : 0;
        const double traces = double(std::max(1, p.receiverCount)) * std::min(p.maxSteps, host::maxBatch) * 2 * 8;
        return int64_t(n * b * (sets * fc + 14 + 2 * L) + sets * b * cpml + traces + allowance);
    }
    const auto &p = s.p3;
    const double n = double((p.nx + 6 + 3) / 4 * 4) * (p.ny + 6) * (p.nz + 6); // pitched rows
    const double b = p.precision == SWL_FP32 ? 4 : 8, sets = p.precision == SWL_FP32 ? 6 : 4;
    const double receivers = double(std::max(1, p.receiverCountX)) * std::max(1, p.receiverCountY);
    const double traces = receivers * std::min(p.maxSteps, host::maxBatch) * 3 * 8;
    const int L = p.attenuation.enabled ? p.attenuation.mechanisms : 0; // GSLS: 6 memory fields and 2 strengths each
    const double material = (p.layered || L) ? 3 : 0;
    return int64_t(n * b * (sets * (9 + 6 * L) + 9 + 5 + material + 2 * L + (p.sourceKind == 1 ? 3 : 0)) + traces + allowance);
}

class Server {
  public:
    explicit Server(const swl_server_config &c) : cfg_(c), t0_(std::chrono::steady_clock::now()) {
        device_ = selectDevice(c.device);
        if (device_ < 0) throw Failure(SWL_ERR_UNAVAILABLE, "no usable sm_100 CUDA device for the server");
        if (cfg_.batch_steps <= 0) cfg_.batch_steps = 64;
        if (cfg_.build_threads <= 0) cfg_.build_threads = 4;
        if (cfg_.scheduler_threads <= 0) cfg_.scheduler_threads = 4;
        budget_ = cfg_.memory_budget;
        if (budget_ <= 0) {
            DeviceScope scope(device_);
            std::size_t freeB = 0, totalB = 0;
            check(cudaMemGetInfo(&freeB, &totalB), "query device memory");
            budget_ = int64_t(0.85 * double(freeB));
        }
        for (int t = 0; t < cfg_.build_threads; ++t) builders_.emplace_back([this] { buildLoop(); });
        for (int t = 0; t < cfg_.scheduler_threads; ++t) loops_.emplace_back([this] { schedule(); });
        if (cfg_.persistent) loops_.emplace_back([this] { queueLoop(); });
        reaper_ = std::thread([this] { reapLoop(); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cvBuild_.notify_all();
        cvWork_.notify_all();
        cvDone_.notify_all();
        cvReap_.notify_all();
        for (auto &t : builders_) t.join();
        for (auto &t : loops_) t.join();
        reaper_.join();
    }
    int64_t submit(std::shared_ptr<Shot> s) {
        std::lock_guard<std::mutex> g(mu_);
        s->id = nextId_++;
        s->submit = now();
        shots_[s->id] = s;
        queue_.push_back(s->id);
        cvWork_.notify_all();
        return s->id;
    }
    swl_shot_status status(int64_t id) {
        std::lock_guard<std::mutex> g(mu_);
        const auto s = find(id);
        swl_shot_status o{};
        o.id = id, o.dim = s->dim, o.state = s->state, o.submit_s = s->submit, o.start_s = s->start, o.finish_s = s->finish;
        o.run_s = s->run;
        o.resident_bytes = s->bytes;
        if (s->state >= SWL_SHOT_RUNNING || s->state == SWL_SHOT_FAILED) {
            o.steps_done = s->steps(), o.total_steps = s->total();
            if (s->dim == 2 && s->s2) o.receivers = int32_t(s->s2->vx.size()), o.samples = s->s2->vx.empty() ? 0 : int64_t(s->s2->vx.front().size());
            if (s->dim == 3 && s->s3) o.receivers = int32_t(s->s3->rec[0].size()), o.samples = int64_t(s->s3->step) + 1;
        }
        std::snprintf(o.error, sizeof(o.error), "%s", s->error.c_str());
        return o;
    }
    int64_t nextFinished(int timeoutMs) {
        std::unique_lock<std::mutex> g(mu_);
        cvDone_.wait_for(g, std::chrono::milliseconds(std::max(0, timeoutMs)), [&] { return !unreported_.empty() || stop_; });
        if (unreported_.empty()) return -1;
        const int64_t id = unreported_.front();
        unreported_.pop_front();
        return id;
    }
    void records(int64_t id, double *vx, double *vy, double *vz) {
        std::lock_guard<std::mutex> g(mu_);
        const auto s = find(id);
        if (s->state != SWL_SHOT_DONE && s->state != SWL_SHOT_FAILED) throw Failure(SWL_ERR_STATE, "shot has not finished");
        const auto copy = [](const std::vector<std::vector<double>> &src, double *dst) {
            if (!dst) return;
            std::size_t at = 0;
            for (const auto &v : src) std::copy(v.begin(), v.end(), dst + at), at += v.size();
        };
        if (s->dim == 2 && s->s2) copy(s->s2->vx, vx), copy(s->s2->vz, vz);
        if (s->dim == 3 && s->s3) copy(s->s3->rec[0], vx), copy(s->s3->rec[1], vy), copy(s->s3->rec[2], vz);
    }
    void release(int64_t id) {
        std::lock_guard<std::mutex> g(mu_);
        const auto s = find(id);
        if (s->state != SWL_SHOT_DONE && s->state != SWL_SHOT_FAILED) throw Failure(SWL_ERR_STATE, "shot has not finished");
        shots_.erase(id);
    }
    void drain() {
        std::unique_lock<std::mutex> g(mu_);
        cvDone_.wait(g, [&] { return stop_ || finished_ == submittedCount(); });
    }
    swl_server_stats stats() {
        std::lock_guard<std::mutex> g(mu_);
        swl_server_stats o{};
        for (const auto &kv : shots_) {
            const int st = kv.second->state;
            o.queued += st == SWL_SHOT_QUEUED, o.building += st == SWL_SHOT_BUILDING, o.running += st == SWL_SHOT_RUNNING;
            o.done += st == SWL_SHOT_DONE, o.failed += st == SWL_SHOT_FAILED;
        }
        o.peak_running = peakRunning_, o.resident_bytes = used_, o.peak_resident_bytes = peakUsed_, o.memory_budget = budget_;
        return o;
    }

  private:
    swl_server_config cfg_;
    int device_{};
    int64_t budget_{}, used_{}, peakUsed_{};
    std::chrono::steady_clock::time_point t0_;
    std::mutex mu_;
    std::condition_variable cvWork_, cvDone_, cvBuild_, cvReap_;
    std::deque<std::shared_ptr<Shot>> reap_; // finished shots whose engines are still to be destroyed
    std::thread reaper_;
    std::deque<int64_t> queue_, unreported_;
    std::deque<std::shared_ptr<Shot>> toBuild_, built_, built2d_; // built2d_: 2D shots for the persistent form
    std::map<int64_t, std::shared_ptr<Shot>> shots_;
    int64_t nextId_{}, finished_{}, building_{};
    int running_{}, peakRunning_{};
    bool stop_{false};
    std::vector<std::thread> builders_;
    std::vector<std::thread> loops_;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count(); }
    int64_t submittedCount() const { return nextId_; }
    std::shared_ptr<Shot> find(int64_t id) {
        const auto it = shots_.find(id);
        if (it == shots_.end()) throw Failure(SWL_ERR_INVALID, "unknown shot id");
        return it->second;
    }
    // caller holds mu_
    // `release`: the shot holds no engine, so its reserved bytes are free now (otherwise the reaper
    // frees them once the engine is destroyed).
    void finishShot(const std::shared_ptr<Shot> &s, int state, const std::string &error, bool release = true) {
        s->state = state;
        s->error = error;
        s->finish = now();
        if (release) used_ -= s->bytes;
        ++finished_;
        unreported_.push_back(s->id);
        cvDone_.notify_all();
        cvWork_.notify_all();
    }
    void buildLoop() {
        for (;;) {
            std::shared_ptr<Shot> s;
            {
                std::unique_lock<std::mutex> g(mu_);
                cvBuild_.wait(g, [&] { return stop_ || !toBuild_.empty(); });
                if (stop_) return;
                s = toBuild_.front();
                toBuild_.pop_front();
            }
            std::string error;
            try { // host FP64 model build, then the engine on its own stream
                if (s->dim == 2) {
                    auto x = std::make_unique<Session2D>();
                    x->params = s->p2;
                    x->params.segmentRule = true; // built while other shots run: no timing runs
                    x->create(device_);
                    s->s2 = std::move(x);
                } else {
                    auto x = std::make_unique<Session3D>();
                    x->params = s->p3;
                    x->create(device_);
                    s->s3 = std::move(x);
                }
            } catch (const std::exception &e) {
                error = e.what();
            }
            std::lock_guard<std::mutex> g(mu_);
            --building_;
            if (!error.empty()) finishShot(s, SWL_SHOT_FAILED, error);
            else {
                const int64_t actual = (s->dim == 2 ? swl2d_resident_bytes(s->s2->engine) : swl3d_resident_bytes(s->s3->engine)) + (16ll << 20);
                used_ += actual - s->bytes;
                s->bytes = actual;
                peakUsed_ = std::max(peakUsed_, used_);
                const bool queued = s->dim == 2 && (cfg_.persistent == 1 || (cfg_.persistent == 2 && s->s2->model.mechanisms == 0));
                (queued ? built2d_ : built_).push_back(s);
                cvWork_.notify_all();
            }
        }
    }
    void reapLoop() {
        for (;;) {
            std::shared_ptr<Shot> s;
            {
                std::unique_lock<std::mutex> g(mu_);
                cvReap_.wait(g, [&] { return stop_ || !reap_.empty(); });
                if (reap_.empty()) return; // stopping, nothing left
                s = reap_.front();
                reap_.pop_front();
            }
            if (s->s2 && s->s2->engine) swl2d_destroy(s->s2->engine), s->s2->engine = nullptr;
            if (s->s3 && s->s3->engine) swl3d_destroy(s->s3->engine), s->s3->engine = nullptr;
            std::lock_guard<std::mutex> g(mu_);
            used_ -= s->bytes;
            cvWork_.notify_all();
        }
    }
    // Admission in arrival order; caller holds mu_.
    void admit(int running) {
        while (!queue_.empty()) {
            const auto s = shots_[queue_.front()];
            const int64_t need = estimate(*s);
            const int active = running + int(building_);
            if (cfg_.max_active > 0 && active >= cfg_.max_active) break;
            if (used_ + need > budget_) {
                if (active > 0) break; // wait for memory to free up
                if (need > budget_) {   // can never fit
                    queue_.pop_front();
                    finishShot(s, SWL_SHOT_FAILED, "request exceeds the server's device-memory budget");
                    continue;
                }
            }
            queue_.pop_front();
            s->state = SWL_SHOT_BUILDING;
            s->start = now();
            s->bytes = need;
            used_ += need;
            peakUsed_ = std::max(peakUsed_, used_);
            ++building_;
            toBuild_.push_back(s);
            cvBuild_.notify_one();
        }
    }
    // One scheduler thread: it takes built shots (one per pass, so the shots spread over the
    // threads) and drives the ones it took -- poll, record, relaunch -- until they finish.
    void schedule() {
        std::vector<std::shared_ptr<Shot>> running;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                if (stop_) break;
                if (!built_.empty()) {
                    built_.front()->state = SWL_SHOT_RUNNING;
                    built_.front()->run = now();
                    running.push_back(built_.front());
                    built_.pop_front();
                    ++running_;
                }
                peakRunning_ = std::max(peakRunning_, running_);
                admit(running_);
            }
            bool progressed = false;
            for (std::size_t i = 0; i < running.size();) {
                auto &s = running[i];
                bool finished = false;
                std::string error;
                try {
                    if (s->dim == 2) {
                        auto &x = *s->s2;
                        if (x.inflight) {
                            if (x.pollBatch(false)) progressed = true;
                        }
                        if (!x.inflight) {
                            if (x.completed()) finished = true;
                            else if (x.launchBatch(cfg_.batch_steps)) progressed = true;
                        }
                    } else {
                        auto &x = *s->s3;
                        if (x.inflight) {
                            if (x.pollBatch(false)) progressed = true;
                        }
                        if (!x.inflight) {
                            if (x.completed()) finished = true;
                            else if (x.launchBatch(cfg_.batch_steps)) progressed = true;
                        }
                    }
                } catch (const std::exception &e) {
                    error = e.what();
                    finished = true;
                }
                if (finished) {
                    // The records stay with the shot.  Its engine is destroyed by the reaper thread:
                    // freeing device memory waits for the whole device, which would stall the other
                    // shots' batches if this loop did it.
                    std::lock_guard<std::mutex> g(mu_);
                    --running_;
                    finishShot(s, error.empty() ? SWL_SHOT_DONE : SWL_SHOT_FAILED, error, false);
                    reap_.push_back(s);
                    cvReap_.notify_one();
                    running.erase(running.begin() + i);
                    progressed = true;
                    continue;
                }
                ++i;
            }
            if (!progressed) {
                std::unique_lock<std::mutex> g(mu_);
                cvWork_.wait_for(g, std::chrono::microseconds(running.empty() ? 2000 : 100));
            }
        }
        for (auto &s : running) { // abandoned on destruction
            if (s->s2 && s->s2->engine) swl2d_destroy(s->s2->engine), s->s2->engine = nullptr;
            if (s->s3 && s->s3->engine) swl3d_destroy(s->s3->engine), s->s3->engine = nullptr;
        }
    }
    // The persistent form's thread: rounds of one multi-shot launch per (precision, mechanisms).
    struct Group {
        swl2d_queue *queue{};
        std::vector<std::shared_ptr<Shot>> shots; // the shots of the launch in flight
        bool inflight{false};
    };
    void finishRunning(const std::shared_ptr<Shot> &s, const std::string &error) {
        std::lock_guard<std::mutex> g(mu_);
        --running_;
        finishShot(s, error.empty() ? SWL_SHOT_DONE : SWL_SHOT_FAILED, error, false);
        reap_.push_back(s);
        cvReap_.notify_one();
    }
    void queueLoop() {
        std::map<std::pair<int, int>, Group> groups;
        std::vector<std::shared_ptr<Shot>> running;
        std::map<int64_t, std::string> failed; // shots whose launch went wrong
        const auto kindOf = [](const Shot &s) { return std::make_pair(s.s2->params.precision, s.s2->model.mechanisms); };
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                if (stop_) break;
                while (!built2d_.empty()) {
                    built2d_.front()->state = SWL_SHOT_RUNNING;
                    built2d_.front()->run = now();
                    running.push_back(built2d_.front());
                    built2d_.pop_front();
                    ++running_;
                }
                peakRunning_ = std::max(peakRunning_, running_);
                admit(running_);
            }
            bool progressed = false;
            for (auto &[kind, grp] : groups) { // completed launches: record each shot's batch
                if (!grp.inflight) continue;
                int32_t done = 0;
                const swl_status st = swl2d_queue_query(grp.queue, &done);
                const std::string why = st == SWL_OK ? std::string() : std::string(swl_last_error());
                if (st == SWL_OK && !done) continue;
                if (st != SWL_OK) swl2d_queue_wait(grp.queue); // settle the launch
                for (auto &s : grp.shots) {
                    try {
                        s->s2->pollBatch(true);
                    } catch (const std::exception &e) {
                        failed[s->id] = e.what();
                    }
                    if (!why.empty()) failed.emplace(s->id, why);
                }
                grp.shots.clear();
                grp.inflight = false;
                progressed = true;
            }
            for (std::size_t i = 0; i < running.size();) { // finished shots
                auto &s = running[i];
                const auto f = failed.find(s->id);
                if (!s->s2->inflight && (f != failed.end() || s->s2->completed())) {
                    finishRunning(s, f == failed.end() ? std::string() : f->second);
                    if (f != failed.end()) failed.erase(f);
                    running.erase(running.begin() + i);
                    progressed = true;
                    continue;
                }
                ++i;
            }
            std::map<std::pair<int, int>, std::vector<std::shared_ptr<Shot>>> ready;
            for (auto &s : running)
                if (!s->s2->inflight) ready[kindOf(*s)].push_back(s);
            for (auto &[kind, shots] : ready) { // one launch per idle kind
                Group &grp = groups[kind];
                if (grp.inflight) continue;
                if (!grp.queue && (swl2d_queue_create(device_, kind.first, &grp.queue) != SWL_OK ||
                                   swl2d_queue_limit(grp.queue, cfg_.persistent_ctas) != SWL_OK)) {
                    const std::string why = swl_last_error();
                    for (auto &s : shots) failed[s->id] = why;
                    progressed = true;
                    continue;
                }
                std::vector<swl2d_engine *> engines;
                std::vector<int32_t> first, count;
                std::vector<double> dt, freq, scale, growth;
                for (auto &s : shots) {
                    int32_t f = 0;
                    double d = 0, fr = 0, sc = 0, gr = 0;
                    int n = 0;
                    try {
                        n = s->s2->queueBatch(cfg_.batch_steps, f, d, fr, sc, gr);
                    } catch (const std::exception &e) {
                        failed[s->id] = e.what();
                    }
                    if (n <= 0) continue;
                    grp.shots.push_back(s);
                    engines.push_back(s->s2->engine), first.push_back(f), count.push_back(n);
                    dt.push_back(d), freq.push_back(fr), scale.push_back(sc), growth.push_back(gr);
                }
                if (engines.empty()) continue;
                if (swl2d_queue_launch(grp.queue, engines.data(), int32_t(engines.size()), first.data(), count.data(), dt.data(),
                                       freq.data(), scale.data(), growth.data()) != SWL_OK) {
                    const std::string why = swl_last_error();
                    for (auto &s : grp.shots) s->s2->inflight = 0, failed[s->id] = why;
                    grp.shots.clear();
                } else {
                    grp.inflight = true;
                }
                progressed = true;
            }
            if (!progressed) {
                std::unique_lock<std::mutex> g(mu_);
                cvWork_.wait_for(g, std::chrono::microseconds(running.empty() ? 2000 : 100));
            }
        }
        for (auto &[kind, grp] : groups) // abandoned on destruction: let the launches end first
            if (grp.queue) swl2d_queue_wait(grp.queue), swl2d_queue_destroy(grp.queue);
        for (auto &s : running)
            if (s->s2 && s->s2->engine) swl2d_destroy(s->s2->engine), s->s2->engine = nullptr;
    }
};

// Worst-fit placement (include/swl_fleet.h): the slot with the most budget left after its
// charges, lower slot on ties; -1 when the charge exceeds every slot's whole budget.
int chooseSlot(int n, const int64_t *budgets, const int64_t *charged, int64_t charge) {
    int best = -1;
    int64_t bestLeft = 0;
    for (int d = 0; d < n; ++d) {
        if (charge > budgets[d]) continue; // can never run there
        const int64_t left = budgets[d] - charged[d];
        if (best < 0 || left > bestLeft) best = d, bestLeft = left;
    }
    return best;
}

// One request loop per device and a front that places each request by budget.  The front keeps
// each shot's charge against its slot until the shot's server reports it finished.
class Fleet {
  public:
    explicit Fleet(const swl_fleet_config &c) {
        std::vector<int> devices;
        if (c.n_devices > 0) {
            if (c.n_devices > SWL_FLEET_MAX_DEVICES) throw Failure(SWL_ERR_INVALID, "too many fleet devices");
            devices.assign(c.devices, c.devices + c.n_devices);
        } else {
            int n = 0;
            if (cudaGetDeviceCount(&n) != cudaSuccess) cudaGetLastError(), n = 0;
            for (int d = 0; d < n && int(devices.size()) < SWL_FLEET_MAX_DEVICES; ++d) {
                cudaDeviceProp pr{};
                if (cudaGetDeviceProperties(&pr, d) == cudaSuccess && pr.major == 10) devices.push_back(d);
            }
        }
        if (devices.empty()) throw Failure(SWL_ERR_UNAVAILABLE, "no usable sm_100 CUDA device for the fleet");
        for (int d : devices) {
            if (selectDevice(d) != d) throw Failure(SWL_ERR_UNAVAILABLE, "fleet device " + std::to_string(d) + " is not usable");
            swl_server_config sc = c.server;
            sc.device = d;
            servers_.push_back(std::make_unique<Server>(sc));
            devices_.push_back(d);
            budgets_.push_back(servers_.back()->stats().memory_budget);
        }
    }
    int size() const { return int(servers_.size()); }
    int device(int slot) const { return slot >= 0 && slot < size() ? devices_[slot] : -1; }
    int64_t submit(std::shared_ptr<Shot> s, int &slot) {
        std::lock_guard<std::mutex> g(mu_);
        const int64_t charge = estimate(*s);
        refresh();
        std::vector<int64_t> charged(size(), 0);
        for (const auto &kv : shots_)
            if (!kv.second.done) charged[kv.second.slot] += kv.second.charge;
        slot = chooseSlot(size(), budgets_.data(), charged.data(), charge);
        if (slot < 0)
            throw Failure(SWL_ERR_MEMORY, "request needs " + std::to_string(charge) + " device bytes, more than any fleet device's budget");
        const int64_t local = servers_[slot]->submit(std::move(s));
        const int64_t id = next_++;
        shots_[id] = Entry{slot, local, charge, false};
        return id;
    }
    swl_shot_status status(int64_t id, int &slot) {
        const Entry e = entry(id);
        slot = e.slot;
        swl_shot_status o = servers_[e.slot]->status(e.local);
        o.id = id;
        return o;
    }
    void records(int64_t id, double *vx, double *vy, double *vz) {
        const Entry e = entry(id);
        servers_[e.slot]->records(e.local, vx, vy, vz);
    }
    void release(int64_t id) {
        const Entry e = entry(id);
        servers_[e.slot]->release(e.local);
        std::lock_guard<std::mutex> g(mu_);
        shots_.erase(id);
    }
    void drain() {
        for (auto &sv : servers_) sv->drain();
    }
    swl_server_stats stats(int slot, int64_t &charged) {
        if (slot < 0 || slot >= size()) throw Failure(SWL_ERR_INVALID, "fleet slot out of range");
        std::lock_guard<std::mutex> g(mu_);
        refresh();
        charged = 0;
        for (const auto &kv : shots_)
            if (!kv.second.done && kv.second.slot == slot) charged += kv.second.charge;
        return servers_[slot]->stats();
    }

  private:
    struct Entry {
        int slot;
        int64_t local, charge;
        bool done;
    };
    Entry entry(int64_t id) {
        std::lock_guard<std::mutex> g(mu_);
        const auto it = shots_.find(id);
        if (it == shots_.end()) throw Failure(SWL_ERR_INVALID, "unknown fleet shot id");
        return it->second;
    }
    // Finished shots stop counting against their device (caller holds mu_).
    void refresh() {
        for (auto &kv : shots_) {
            if (kv.second.done) continue;
            const int st = servers_[kv.second.slot]->status(kv.second.local).state;
            kv.second.done = st == SWL_SHOT_DONE || st == SWL_SHOT_FAILED;
        }
    }
    std::vector<std::unique_ptr<Server>> servers_;
    std::vector<int> devices_;
    std::vector<int64_t> budgets_;
    std::map<int64_t, Entry> shots_;
    int64_t next_{0};
    std::mutex mu_;
};

} // namespace swl::host

struct swl_server : swl::host::Server {
    using Server::Server;
};
struct swl_fleet : swl::host::Fleet {
    using Fleet::Fleet;
};

extern "C" {
void swl_server_config_default(swl_server_config *c) {
    if (!c) return;
    *c = swl_server_config{};
    c->device = -1, c->memory_budget = 0, c->max_active = 0, c->batch_steps = 64, c->build_threads = 4;
    c->scheduler_threads = 4;
    c->persistent = 0;
    c->persistent_ctas = -1;
}
swl_status swl_server_create(const swl_server_config *c, swl_server **out) {
    return swl::host::guard([&] {
        if (!c || !out) throw swl::host::Failure(SWL_ERR_INVALID, "config and out are required");
        *out = new swl_server(*c);
    });
}
void swl_server_destroy(swl_server *s) { delete s; }
swl_status swl_server_submit2d(swl_server *s, const swl_params2d *p, int64_t *id) {
    return swl::host::guard([&] {
        if (!s || !p || !id) throw swl::host::Failure(SWL_ERR_INVALID, "server, params and id are required");
        auto shot = std::make_shared<swl::host::Shot>();
        shot->dim = 2;
        shot->p2 = swl::host::toParams(*p);
        *id = s->submit(shot);
    });
}
swl_status swl_server_submit3d(swl_server *s, const swl_params3d *p, int64_t *id) {
    return swl::host::guard([&] {
        if (!s || !p || !id) throw swl::host::Failure(SWL_ERR_INVALID, "server, params and id are required");
        auto shot = std::make_shared<swl::host::Shot>();
        shot->dim = 3;
        shot->p3 = swl::host::toParams(*p);
        *id = s->submit(shot);
    });
}
swl_status swl_server_status(swl_server *s, int64_t id, swl_shot_status *out) {
    return swl::host::guard([&] {
        if (!s || !out) throw swl::host::Failure(SWL_ERR_INVALID, "server and out are required");
        *out = s->status(id);
    });
}
swl_status swl_server_next_finished(swl_server *s, int32_t timeoutMs, int64_t *id) {
    return swl::host::guard([&] {
        if (!s || !id) throw swl::host::Failure(SWL_ERR_INVALID, "server and id are required");
        *id = s->nextFinished(timeoutMs);
    });
}
swl_status swl_server_records(swl_server *s, int64_t id, double *vx, double *vy, double *vz) {
    return swl::host::guard([&] {
        if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "server is null");
        s->records(id, vx, vy, vz);
    });
}
swl_status swl_server_release(swl_server *s, int64_t id) {
    return swl::host::guard([&] {
        if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "server is null");
        s->release(id);
    });
}
swl_status swl_server_drain(swl_server *s) {
    return swl::host::guard([&] {
        if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "server is null");
        s->drain();
    });
}
swl_status swl_request_bytes2d(const swl_params2d *p, int64_t *bytes) {
    return swl::host::guard([&] {
        if (!p || !bytes) throw swl::host::Failure(SWL_ERR_INVALID, "params and bytes are required");
        swl::host::Shot shot;
        shot.dim = 2;
        shot.p2 = swl::host::toParams(*p);
        *bytes = swl::host::estimate(shot);
    });
}
swl_status swl_request_bytes3d(const swl_params3d *p, int64_t *bytes) {
    return swl::host::guard([&] {
        if (!p || !bytes) throw swl::host::Failure(SWL_ERR_INVALID, "params and bytes are required");
        swl::host::Shot shot;
        shot.dim = 3;
        shot.p3 = swl::host::toParams(*p);
        *bytes = swl::host::estimate(shot);
    });
}
int32_t swl_fleet_choose(int32_t n, const int64_t *budgets, const int64_t *charged, int64_t charge) {
    if (n <= 0 || !budgets || !charged || charge < 0) return -1;
    return swl::host::chooseSlot(n, budgets, charged, charge);
}
void swl_fleet_config_default(swl_fleet_config *c) {
    if (!c) return;
    *c = swl_fleet_config{};
    swl_server_config_default(&c->server);
}
swl_status swl_fleet_create(const swl_fleet_config *c, swl_fleet **out) {
    return swl::host::guard([&] {
        if (!c || !out) throw swl::host::Failure(SWL_ERR_INVALID, "config and out are required");
        *out = new swl_fleet(*c);
    });
}
void swl_fleet_destroy(swl_fleet *f) { delete f; }
int32_t swl_fleet_size(const swl_fleet *f) { return f ? f->size() : 0; }
int32_t swl_fleet_device(const swl_fleet *f, int32_t slot) { return f ? f->device(slot) : -1; }
swl_status swl_fleet_submit2d(swl_fleet *f, const swl_params2d *p, int64_t *id, int32_t *slot) {
    return swl::host::guard([&] {
        if (!f || !p || !id) throw swl::host::Failure(SWL_ERR_INVALID, "fleet, params and id are required");
        auto shot = std::make_shared<swl::host::Shot>();
        shot->dim = 2;
        shot->p2 = swl::host::toParams(*p);
        int sl = -1;
        *id = f->submit(shot, sl);
        if (slot) *slot = sl;
    });
}
swl_status swl_fleet_submit3d(swl_fleet *f, const swl_params3d *p, int64_t *id, int32_t *slot) {
    return swl::host::guard([&] {
        if (!f || !p || !id) throw swl::host::Failure(SWL_ERR_INVALID, "fleet, params and id are required");
        auto shot = std::make_shared<swl::host::Shot>();
        shot->dim = 3;
        shot->p3 = swl::host::toParams(*p);
        int sl = -1;
        *id = f->submit(shot, sl);
        if (slot) *slot = sl;
    });
}
swl_status swl_fleet_status(swl_fleet *f, int64_t id, swl_shot_status *out, int32_t *slot) {
    return swl::host::guard([&] {
        if (!f || !out) throw swl::host::Failure(SWL_ERR_INVALID, "fleet and out are required");
        int sl = -1;
        *out = f->status(id, sl);
        if (slot) *slot = sl;
    });
}
swl_status swl_fleet_records(swl_fleet *f, int64_t id, double *vx, double *vy, double *vz) {
    return swl::host::guard([&] {
        if (!f) throw swl::host::Failure(SWL_ERR_INVALID, "fleet is null");
        f->records(id, vx, vy, vz);
    });
}
swl_status swl_fleet_release(swl_fleet *f, int64_t id) {
    return swl::host::guard([&] {
        if (!f) throw swl::host::Failure(SWL_ERR_INVALID, "fleet is null");
        f->release(id);
    });
}
swl_status swl_fleet_drain(swl_fleet *f) {
    return swl::host::guard([&] {
        if (!f) throw swl::host::Failure(SWL_ERR_INVALID, "fleet is null");
        f->drain();
    });
}
swl_status swl_fleet_stats(swl_fleet *f, int32_t slot, swl_server_stats *out, int64_t *charged) {
    return swl::host::guard([&] {
        if (!f || !out) throw swl::host::Failure(SWL_ERR_INVALID, "fleet and out are required");
        int64_t c = 0;
        *out = f->stats(slot, c);
        if (charged) *charged = c;
    });
}
swl_status swl_server_stats_get(swl_server *s, swl_server_stats *out) {
    return swl::host::guard([&] {
        if (!s || !out) throw swl::host::Failure(SWL_ERR_INVALID, "server and out are required");
        *out = s->stats();
    });
}
} // extern "C"
