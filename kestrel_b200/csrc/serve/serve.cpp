// serve.cpp -- the render server of include/kestrel_serve.h.
//
// Batched mode is a continuous-batching loop on one thread (the scheduler)
// with two host thread pools: one builds arriving jobs' banks and drivers
// (seconds of CPU for a large soundfont), the other prepares every resident
// job's block inputs before a step and consumes its output after. Each step
// renders one block of every resident job with one kc_batch_render. Jobs are
// admitted first come, first served, while a batch slot is free and their
// device-byte estimate fits the budget; a finished job's context is freed
// before the next admission.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/kestrel_serve.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

using Clock = std::chrono::steady_clock;

double since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

// KESTREL_SERVE_TRACE=1: one stderr line per batch step (or per sequential
// job) with the phase times, for following a long run.
bool trace_on() {
    static const bool on = [] {
        const char* v = std::getenv("KESTREL_SERVE_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}

// A fixed set of threads running queued tasks; parallel_for lets the caller
// take part and returns when every index is done.
class Workers {
public:
    explicit Workers(unsigned n) {
        for (unsigned i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
    }
    ~Workers() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    unsigned size() const { return (unsigned)th_.size(); }
    void run(std::function<void()> f) {
        {
            std::lock_guard<std::mutex> g(m_);
            q_.push_back(std::move(f));
        }
        cv_.notify_one();
    }
    void parallel_for(size_t n, const std::function<void(size_t)>& f) {
        if (n == 0) return;
        std::atomic<size_t> next{0};
        std::atomic<size_t> left{n};
        std::mutex dm;
        std::condition_variable dcv;
        auto body = [&] {
            for (size_t i; (i = next.fetch_add(1)) < n;) {
                f(i);
                if (left.fetch_sub(1) == 1) {
                    std::lock_guard<std::mutex> g(dm);
                    dcv.notify_all();
                }
            }
        };
        const size_t helpers = std::min<size_t>(th_.size(), n - 1);
        for (size_t k = 0; k < helpers; ++k) run(body);
        body();
        {
            // Released before the idle wait below: the helper that finished
            // the last index takes this lock to notify, and it must be able
            // to, or it never goes idle.
            std::unique_lock<std::mutex> g(dm);
            dcv.wait(g, [&] { return left.load() == 0; });
        }
        // Helpers may still be inside body() (notifying, or having found no
        // index); wait for them before the locals they use go away.
        std::unique_lock<std::mutex> g2(m_);
        idle_cv_.wait(g2, [&] { return q_.empty() && busy_ == 0; });
    }

private:
    void loop() {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return stop_ || !q_.empty(); });
                if (stop_ && q_.empty()) return;
                f = std::move(q_.front());
                q_.pop_front();
                ++busy_;
            }
            f();
            {
                std::lock_guard<std::mutex> g(m_);
                --busy_;
            }
            idle_cv_.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, idle_cv_;
    std::deque<std::function<void()>> q_;
    unsigned busy_ = 0;
    bool stop_ = false;
};

struct Job {
    uint32_t id = 0;
    const ks_job_spec* spec = nullptr;
    ks_job_result* res = nullptr;
    kh_bank* bank = nullptr;
    kh_driver* drv = nullptr;
    kc_synth* synth = nullptr;
    std::vector<float> out;
    uint64_t est_bytes = 0;
    uint32_t live = 0;
    bool finished = false;
    int status = KC_OK;
    std::string err;
};

void release(Job& j) {
    if (j.synth) kc_synth_destroy(j.synth);
    if (j.drv) kh_driver_destroy(j.drv);
    if (j.bank) kh_bank_destroy(j.bank);
    j.synth = nullptr;
    j.drv = nullptr;
    j.bank = nullptr;
}

// Bank and driver (the bank's samples convert on the GPU when the server
// installed the device resampler).
void setup(Job& j) {
    const auto t0 = Clock::now();
    const ks_job_spec& sp = *j.spec;
    j.bank = kh_bank_synthetic(&sp.bank, &sp.cfg, &sp.opt);
    if (!j.bank) {
        j.status = KC_ERR_INVALID;
        j.err = std::string("bank: ") + kh_last_error();
    } else {
        j.drv = kh_driver_open(&sp.cfg, &sp.opt, j.bank, &sp.midi);
        if (!j.drv) {
            j.status = KC_ERR_INVALID;
            j.err = std::string("driver: ") + kh_last_error();
        }
    }
    if (j.status == KC_OK) {
        const int16_t* pool = nullptr;
        uint64_t pool_len = 0;
        const kc_region_params* params = nullptr;
        uint32_t n_params = 0;
        kh_bank_pool(j.bank, &pool, &pool_len);
        kh_bank_params(j.bank, &params, &n_params);
        if (int rc = kc_estimate_device_bytes(&sp.cfg, pool_len, n_params, &j.est_bytes)) {
            j.status = rc;
            j.err = kc_last_error();
        }
    }
    j.out.assign((size_t)sp.cfg.block_frames * 2, 0.0f);
    j.res->setup_s = since(t0);
}

// The context on the device; called on the scheduler thread.
int create(Job& j) {
    const int16_t* pool = nullptr;
    uint64_t pool_len = 0;
    const kc_region_params* params = nullptr;
    uint32_t n_params = 0;
    kh_bank_pool(j.bank, &pool, &pool_len);
    kh_bank_params(j.bank, &params, &n_params);
    const int rc = kc_synth_create(&j.spec->cfg, pool, pool_len, params, n_params, kh_bank_regions(j.bank),
                                   kh_bank_max_sample_len(j.bank), &j.synth);
    if (rc) {
        j.status = rc;
        j.err = kc_last_error();
        return rc;
    }
    // Charge the most the context can grow to (its spawn buffer follows the
    // largest block), never less than what it holds now.
    j.res->device_bytes = std::max<uint64_t>(j.est_bytes, kc_synth_device_bytes(j.synth));
    return KC_OK;
}

// Driver::next_block up to spawn, handed to the context in the reference's
// call order (src/driver.rs:531-588).
int prepare(Job& j) {
    kh_block b{};
    if (kh_driver_prepare(j.drv, j.live, &b)) return fail(KC_ERR_INVALID, std::string("prepare: ") + kh_last_error());
    for (uint32_t i = 0; i < b.n_variants; ++i) {
        uint32_t idx = 0;
        const kc_region_params* data = nullptr;
        size_t n = 0;
        if (kh_driver_variant(j.drv, i, &idx, &data, &n)) return fail(KC_ERR_INVALID, kh_last_error());
        if (int rc = kc_set_params_variant(j.synth, idx, data, n)) return fail(rc, kc_last_error());
    }
    if (int rc = kc_set_gates(j.synth, b.gates, b.n_gates)) return fail(rc, kc_last_error());
    if (int rc = kc_set_channels(j.synth, b.chan, b.n_chan, b.bend, b.gain, b.variant)) return fail(rc, kc_last_error());
    if (int rc = kc_spawn(j.synth, b.cmds, b.n_cmds)) return fail(rc, kc_last_error());
    return KC_OK;
}

// After the block: stats, accounting, hash, the rest of next_block.
int finish(Job& j, const ks_server_config& sc, double now) {
    kc_block_stats st{};
    kc_stats(j.synth, &st);
    uint32_t rendered = 0;
    kc_last_block_voices(j.synth, &rendered);
    ks_job_result& r = *j.res;
    if (r.blocks == 0) r.first_block_s = now;
    r.voice_samples += (uint64_t)rendered * j.spec->cfg.block_frames;
    r.out_hash = ks_hash_block(r.out_hash, j.out.data(), j.out.size());
    r.max_live = std::max<uint32_t>(r.max_live, (uint32_t)std::min<uint64_t>(st.active_voices, 0xFFFFFFFFu));
    r.peak = std::max(r.peak, st.peak);
    if (sc.on_block) sc.on_block(sc.user, j.id, r.blocks, j.out.data(), j.out.size());
    r.blocks += 1;
    j.live = (uint32_t)std::min<uint64_t>(st.active_voices, 0xFFFFFFFFu);
    int more = 0;
    if (kh_driver_finish(j.drv, st.active_voices, &more)) return fail(KC_ERR_INVALID, kh_last_error());
    if (!more || (j.spec->max_blocks && r.blocks >= j.spec->max_blocks)) j.finished = true;
    return KC_OK;
}

// Device milliseconds of every block a job's context rendered (its per-pass
// event timings, switched on when the context was created).
double device_ms(Job& j) {
    if (!j.synth) return 0.0;
    double ms[8] = {};  // kc_timings_total fills one entry per pass (five)
    uint64_t blocks = 0;
    if (kc_timings_total(j.synth, ms, 8, &blocks)) return 0.0;
    double t = 0.0;
    for (double x : ms) t += x;
    return t;
}

bool same_batch_variant(const kc_config& a, const kc_config& b) {
    const uint32_t va = a.voices_per_lane == 2 ? 2 : 1, vb = b.voices_per_lane == 2 ? 2 : 1;
    const uint32_t ra = a.sort_radix_bits ? a.sort_radix_bits : 8, rb = b.sort_radix_bits ? b.sort_radix_bits : 8;
    return a.device == b.device && a.block_frames == b.block_frames && a.interpolation == b.interpolation &&
           (a.strict_fp != 0) == (b.strict_fp != 0) && a.mix_mode == b.mix_mode && va == vb && ra == rb;
}

int serve_sequential(const ks_server_config& sc, std::vector<Job>& jobs, const std::vector<uint32_t>& order,
                     ks_run_stats& rs, Clock::time_point t0) {
    for (uint32_t id : order) {
        Job& j = jobs[id];
        if (sc.realtime_arrivals) {
            const double wait = j.spec->arrival_s - since(t0);
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
        }
        setup(j);
        rs.setup_s += j.res->setup_s;
        if (j.status == KC_OK && create(j) == KC_OK) kc_set_profile(j.synth, 1);
        j.res->admit_s = since(t0);
        rs.max_resident = 1;
        rs.peak_device_bytes = std::max(rs.peak_device_bytes, j.res->device_bytes);
        while (j.status == KC_OK && !j.finished) {
            if (int rc = prepare(j)) {
                j.status = rc;
                j.err = g_err;
                break;
            }
            if (int rc = kc_render(j.synth, j.out.data(), j.out.size())) {
                j.status = rc;
                j.err = kc_last_error();
                break;
            }
            if (int rc = finish(j, sc, since(t0))) {
                j.status = rc;
                j.err = g_err;
            }
            rs.steps += 1;
        }
        j.res->done_s = since(t0);
        j.res->status = j.status;
        rs.gpu_ms += device_ms(j);
        if (trace_on())
            std::fprintf(stderr, "[serve] t=%.3f job=%u blocks=%llu setup_s=%.3f run_s=%.3f status=%d\n", since(t0), j.id,
                         (unsigned long long)j.res->blocks, j.res->setup_s, j.res->done_s - j.res->admit_s, j.status);
        release(j);
    }
    return KC_OK;
}

// The plain path on several host threads at once: each thread takes the next
// job in arrival order, builds its bank and driver, waits until the job's
// device-byte bound fits the budget beside the jobs already running, and
// renders it to completion through kc_render on its own context (and so its
// own stream). Jobs run side by side on the device, one context each, with
// no batching: the baseline that shows what batching adds beyond running
// many contexts at once.
int serve_parallel(const ks_server_config& sc, std::vector<Job>& jobs, const std::vector<uint32_t>& order,
                   ks_run_stats& rs, Clock::time_point t0) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned n_threads = std::min<unsigned>(sc.host_threads ? sc.host_threads : hw, (unsigned)jobs.size());
    rs.host_threads = n_threads;
    uint64_t budget = sc.vram_budget;
    if (!budget) {
        uint64_t f = 0, t = 0;
        if (int rc = kc_device_memory((int)sc.device, &f, &t)) return fail(rc, kc_last_error());
        const uint64_t reserve = 8ull << 30;
        budget = f > reserve ? f - reserve : f / 2;
    }
    std::mutex m;
    std::condition_variable cv;
    size_t next = 0;
    uint64_t used = 0;
    uint32_t running = 0;
    auto worker = [&] {
        for (;;) {
            uint32_t id;
            {
                std::lock_guard<std::mutex> g(m);
                if (next >= order.size()) return;
                id = order[next++];
            }
            Job& j = jobs[id];
            if (sc.realtime_arrivals) {
                const double wait = j.spec->arrival_s - since(t0);
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
            }
            setup(j);
            {
                std::unique_lock<std::mutex> g(m);
                rs.setup_s += j.res->setup_s;
                if (j.status == KC_OK && j.est_bytes > budget) {
                    j.status = KC_ERR_OOM;
                    j.err = "job needs more device memory than the budget";
                }
                if (j.status == KC_OK) {
                    cv.wait(g, [&] { return running == 0 || used + j.est_bytes <= budget; });
                    used += j.est_bytes;
                    ++running;
                    rs.max_resident = std::max(rs.max_resident, running);
                    rs.peak_device_bytes = std::max(rs.peak_device_bytes, used);
                }
            }
            const bool admitted = j.status == KC_OK;
            if (admitted && create(j) == KC_OK) kc_set_profile(j.synth, 1);
            j.res->admit_s = since(t0);
            uint64_t blocks = 0;
            while (j.status == KC_OK && !j.finished) {
                if (int rc = prepare(j)) {
                    j.status = rc;
                    j.err = g_err;
                    break;
                }
                if (int rc = kc_render(j.synth, j.out.data(), j.out.size())) {
                    j.status = rc;
                    j.err = kc_last_error();
                    break;
                }
                if (int rc = finish(j, sc, since(t0))) {
                    j.status = rc;
                    j.err = g_err;
                }
                ++blocks;
            }
            j.res->done_s = since(t0);
            j.res->status = j.status;
            const double ms = device_ms(j);
            release(j);
            {
                std::lock_guard<std::mutex> g(m);
                rs.gpu_ms += ms;
                rs.steps += blocks;
                if (admitted) {
                    used -= std::min(used, j.est_bytes);
                    --running;
                }
            }
            cv.notify_all();
        }
    };
    std::vector<std::thread> th;
    for (unsigned i = 0; i < n_threads; ++i) th.emplace_back(worker);
    for (auto& t : th) t.join();
    return KC_OK;
}

int serve_batched(const ks_server_config& sc, std::vector<Job>& jobs, const std::vector<uint32_t>& order,
                  ks_run_stats& rs, Clock::time_point t0) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned total = sc.host_threads ? sc.host_threads : hw;
    const unsigned n_setup = std::max(1u, total / 4), n_step = std::max(1u, total - n_setup);
    rs.host_threads = n_setup + n_step;
    uint64_t budget = sc.vram_budget;
    if (!budget) {
        uint64_t f = 0, t = 0;
        if (int rc = kc_device_memory((int)sc.device, &f, &t)) return fail(rc, kc_last_error());
        const uint64_t reserve = 8ull << 30;
        budget = f > reserve ? f - reserve : f / 2;
    }
    kc_batch_config bc{};
    kc_batch_config_default(&bc);
    const kc_config& c0 = jobs[order[0]].spec->cfg;
    bc.device = sc.device;
    bc.max_jobs = sc.max_jobs;
    bc.block_frames = c0.block_frames;
    bc.interpolation = c0.interpolation;
    bc.strict_fp = c0.strict_fp;
    bc.mix_mode = c0.mix_mode;
    bc.voices_per_lane = c0.voices_per_lane == 2 ? 2 : 1;
    bc.sort_radix_bits = c0.sort_radix_bits;
    bc.use_graph = sc.use_graph;
    kc_batch* batch = nullptr;
    if (int rc = kc_batch_create(&bc, &batch)) return fail(rc, kc_last_error());

    std::mutex rm;
    std::condition_variable rcv;
    size_t next = 0, completed = 0;
    uint64_t used = 0;
    std::vector<uint32_t> resident;
    std::vector<kc_synth*> synths;
    std::vector<float*> outs;
    std::vector<int> prc;
    // Arrival order is the admission order: a job set up early waits for the
    // ones that arrived before it.
    std::vector<char> set_up(jobs.size(), 0);
    size_t admit_cursor = 0;
    int rc_out = KC_OK;
    // Declared after the state their tasks touch, and joined before it goes.
    auto setup_pool = std::make_unique<Workers>(n_setup);
    auto step_pool = std::make_unique<Workers>(n_step - 1);  // the scheduler thread is a step worker too

    auto retire = [&](Job& j) {
        used -= std::min(used, j.res->device_bytes);
        j.res->done_s = since(t0);
        j.res->status = j.status;
        release(j);
        ++completed;
    };

    while (completed < jobs.size()) {
        const double now = since(t0);
        while (next < order.size() && (!sc.realtime_arrivals || jobs[order[next]].spec->arrival_s <= now)) {
            const uint32_t id = order[next++];
            setup_pool->run([&, id] {
                setup(jobs[id]);
                std::lock_guard<std::mutex> g(rm);
                set_up[id] = 1;
                rcv.notify_all();
            });
        }
        // Admission, first come first served.
        {
            std::unique_lock<std::mutex> g(rm);
            while (admit_cursor < next && set_up[order[admit_cursor]] && resident.size() < sc.max_jobs) {
                Job& j = jobs[order[admit_cursor]];
                if (j.status != KC_OK) {
                    rs.setup_s += j.res->setup_s;
                    j.res->admit_s = since(t0);
                    ++admit_cursor;
                    g.unlock();
                    retire(j);
                    g.lock();
                    continue;
                }
                if (used + j.est_bytes > budget && !resident.empty()) break;
                ++admit_cursor;
                g.unlock();
                rs.setup_s += j.res->setup_s;
                if (j.est_bytes > budget) {
                    j.status = KC_ERR_OOM;
                    j.err = "job needs more device memory than the budget";
                } else {
                    create(j);
                }
                j.res->admit_s = since(t0);
                if (j.status != KC_OK) {
                    retire(j);
                } else {
                    used += j.res->device_bytes;
                    rs.peak_device_bytes = std::max(rs.peak_device_bytes, used);
                    resident.push_back(j.id);
                }
                g.lock();
            }
            if (resident.empty()) {
                if (completed == jobs.size()) break;
                // Nothing to render: wait for a setup to finish or the next arrival.
                double wait = 0.05;
                if (next < order.size() && sc.realtime_arrivals)
                    wait = std::min(wait, std::max(0.0, jobs[order[next]].spec->arrival_s - since(t0)));
                rcv.wait_for(g, std::chrono::duration<double>(wait));
                continue;
            }
        }
        rs.max_resident = std::max<uint32_t>(rs.max_resident, (uint32_t)resident.size());
        const auto t_step = Clock::now();
        // Prepare every resident job's block.
        prc.assign(resident.size(), KC_OK);
        step_pool->parallel_for(resident.size(), [&](size_t k) {
            Job& j = jobs[resident[k]];
            prc[k] = prepare(j);
            if (prc[k]) j.err = g_err;
        });
        synths.clear();
        outs.clear();
        std::vector<uint32_t> stepping;
        for (size_t k = 0; k < resident.size(); ++k) {
            Job& j = jobs[resident[k]];
            if (prc[k]) {
                j.status = prc[k];
                j.finished = true;
                continue;
            }
            stepping.push_back(resident[k]);
            synths.push_back(j.synth);
            outs.push_back(j.out.data());
        }
        if (!stepping.empty()) {
            const int rc = kc_batch_render(batch, synths.data(), (uint32_t)synths.size(), outs.data());
            if (rc) {
                rc_out = fail(rc, kc_last_error());
                for (uint32_t id : stepping) {
                    jobs[id].status = rc;
                    jobs[id].err = g_err;
                    jobs[id].finished = true;
                }
            } else {
                float ms = 0.0f;
                kc_batch_last_ms(batch, &ms);
                rs.gpu_ms += ms;
                rs.steps += 1;
                const double t_done = since(t0);
                step_pool->parallel_for(stepping.size(), [&](size_t k) {
                    Job& j = jobs[stepping[k]];
                    if (int e = finish(j, sc, t_done)) {
                        j.status = e;
                        j.err = g_err;
                        j.finished = true;
                    }
                });
                if (trace_on())
                    std::fprintf(stderr, "[serve] t=%.3f step=%llu resident=%zu gpu_ms=%.2f step_ms=%.2f used_gb=%.2f "
                                 "done=%zu/%zu\n", since(t0), (unsigned long long)rs.steps, stepping.size(), ms,
                                 since(t_step) * 1e3, used / 1e9, completed, jobs.size());
            }
        }
        // Retire finished jobs; their memory is free for the next admission.
        std::vector<uint32_t> keep;
        for (uint32_t id : resident) {
            if (jobs[id].finished) retire(jobs[id]);
            else keep.push_back(id);
        }
        resident.swap(keep);
        if (rc_out) break;
    }
    // Let queued setups finish, then free whatever a failure left behind.
    setup_pool.reset();
    step_pool.reset();
    for (uint32_t id : resident) retire(jobs[id]);
    for (Job& j : jobs) release(j);
    kc_batch_destroy(batch);
    return rc_out;
}

// ---- autotuner ----------------------------------------------------------------

// One block's inputs copied out of the driver.
struct Recorded {
    std::vector<uint32_t> gates, chan;
    std::vector<kc_spawn_cmd> cmds;
    std::vector<std::pair<uint32_t, std::vector<kc_region_params>>> variants;
    int bend = 0, gain = 0, variant = 0;
};

int record_block(kh_driver* drv, uint32_t live, Recorded& r) {
    kh_block b{};
    if (kh_driver_prepare(drv, live, &b)) return fail(KC_ERR_INVALID, std::string("prepare: ") + kh_last_error());
    r.gates.assign(b.gates, b.gates + b.n_gates);
    r.chan.assign(b.chan, b.chan + b.n_chan);
    r.cmds.assign(b.cmds, b.cmds + b.n_cmds);
    r.bend = b.bend;
    r.gain = b.gain;
    r.variant = b.variant;
    r.variants.clear();
    for (uint32_t i = 0; i < b.n_variants; ++i) {
        uint32_t idx = 0;
        const kc_region_params* data = nullptr;
        size_t n = 0;
        if (kh_driver_variant(drv, i, &idx, &data, &n)) return fail(KC_ERR_INVALID, kh_last_error());
        r.variants.emplace_back(idx, std::vector<kc_region_params>(data, data + n));
    }
    return KC_OK;
}

int feed_block(kc_synth* s, const Recorded& r) {
    for (const auto& v : r.variants)
        if (int rc = kc_set_params_variant(s, v.first, v.second.data(), v.second.size())) return fail(rc, kc_last_error());
    if (int rc = kc_set_gates(s, r.gates.data(), r.gates.size())) return fail(rc, kc_last_error());
    if (int rc = kc_set_channels(s, r.chan.data(), r.chan.size(), r.bend, r.gain, r.variant))
        return fail(rc, kc_last_error());
    if (int rc = kc_spawn(s, r.cmds.data(), r.cmds.size())) return fail(rc, kc_last_error());
    return KC_OK;
}

// Render one recorded block; returns the voices it rendered.
int render_recorded(kc_synth* s, const Recorded& r, std::vector<float>& out, uint32_t* rendered) {
    if (int rc = feed_block(s, r)) return rc;
    if (int rc = kc_render(s, out.data(), out.size())) return fail(rc, kc_last_error());
    if (int rc = kc_last_block_voices(s, rendered)) return fail(rc, kc_last_error());
    return KC_OK;
}

struct Owned {
    kh_bank* bank = nullptr;
    kh_driver* drv = nullptr;
    kc_synth* snap = nullptr;
    kc_synth* live = nullptr;
    ~Owned() {
        if (live) kc_synth_destroy(live);
        if (snap) kc_synth_destroy(snap);
        if (drv) kh_driver_destroy(drv);
        if (bank) kh_bank_destroy(bank);
    }
};

// Tune one block length: pre-roll, snapshot, record, replay per candidate.
int tune_block_length(const ks_job_spec& job, uint32_t bf, const std::vector<uint32_t>& vpls,
                      const std::vector<uint32_t>& radices, uint32_t preroll, uint32_t timed,
                      std::vector<ks_tune_result>& out) {
    kc_config cfg = job.cfg;
    cfg.block_frames = bf;
    cfg.voices_per_lane = 0;
    cfg.sort_radix_bits = 0;
    Owned o;
    o.bank = kh_bank_synthetic(&job.bank, &cfg, &job.opt);
    if (!o.bank) return fail(KC_ERR_INVALID, std::string("bank: ") + kh_last_error());
    o.drv = kh_driver_open(&cfg, &job.opt, o.bank, &job.midi);
    if (!o.drv) return fail(KC_ERR_INVALID, std::string("driver: ") + kh_last_error());
    const int16_t* pool = nullptr;
    uint64_t pool_len = 0;
    const kc_region_params* params = nullptr;
    uint32_t n_params = 0;
    kh_bank_pool(o.bank, &pool, &pool_len);
    kh_bank_params(o.bank, &params, &n_params);
    if (int rc = kc_synth_create(&cfg, pool, pool_len, params, n_params, kh_bank_regions(o.bank),
                                 kh_bank_max_sample_len(o.bank), &o.live))
        return fail(rc, kc_last_error());
    std::vector<float> buf((size_t)bf * 2);
    Recorded r;
    uint32_t live = 0, rendered = 0;
    int more = 1;
    kc_block_stats st{};
    for (uint32_t i = 0; i < preroll && more; ++i) {
        if (int rc = record_block(o.drv, live, r)) return rc;
        if (int rc = render_recorded(o.live, r, buf, &rendered)) return rc;
        kc_stats(o.live, &st);
        live = (uint32_t)std::min<uint64_t>(st.active_voices, 0xFFFFFFFFu);
        if (kh_driver_finish(o.drv, st.active_voices, &more)) return fail(KC_ERR_INVALID, kh_last_error());
    }
    if (int rc = kc_synth_clone(o.live, &o.snap)) return fail(rc, kc_last_error());
    std::vector<Recorded> rec;
    // One more block than timed: each candidate renders the first untimed,
    // so its kernels are loaded before the clock starts.
    for (uint32_t i = 0; i < timed + 1 && more; ++i) {
        rec.emplace_back();
        if (int rc = record_block(o.drv, live, rec.back())) return rc;
        if (int rc = render_recorded(o.live, rec.back(), buf, &rendered)) return rc;
        kc_stats(o.live, &st);
        live = (uint32_t)std::min<uint64_t>(st.active_voices, 0xFFFFFFFFu);
        if (kh_driver_finish(o.drv, st.active_voices, &more)) return fail(KC_ERR_INVALID, kh_last_error());
    }
    if (rec.empty()) return fail(KC_ERR_INVALID, "the job ended before any block could be timed");
    for (uint32_t v : vpls) {
        for (uint32_t rb : radices) {
            kc_config c = cfg;
            c.voices_per_lane = v;
            c.sort_radix_bits = rb;
            kc_synth* k = nullptr;
            if (int rc = kc_synth_clone_config(o.snap, &c, &k)) return fail(rc, kc_last_error());
            ks_tune_result res{};
            res.voices_per_lane = v;
            res.sort_radix_bits = rb;
            res.block_frames = bf;
            int rc = KC_OK;
            const size_t first_timed = rec.size() > 1 ? 1 : 0;
            for (size_t i = 0; i < rec.size() && rc == KC_OK; ++i) {
                if (i == first_timed) rc = kc_set_profile(k, 1);
                if (rc == KC_OK) rc = render_recorded(k, rec[i], buf, &rendered);
                if (i >= first_timed) res.voice_samples += (uint64_t)rendered * bf;
            }
            double ms[8] = {};
            uint64_t blocks = 0;
            if (rc == KC_OK && (rc = kc_timings_total(k, ms, 8, &blocks)) != KC_OK) fail(rc, kc_last_error());
            kc_synth_destroy(k);
            if (rc) return rc;
            for (double m : ms) res.device_ms += m;
            res.blocks = (uint32_t)blocks;
            res.voice_samples_per_s = res.device_ms > 0 ? res.voice_samples / (res.device_ms * 1e-3) : 0.0;
            out.push_back(res);
        }
    }
    return KC_OK;
}

}  // namespace

extern "C" {

int ks_autotune(const ks_job_spec* job, const ks_tune_space* space, kc_config* best, ks_tune_result* results,
                uint32_t cap, uint32_t* n) {
    if (!job || !best) return fail(KC_ERR_INVALID, "null argument");
    ks_tune_space sp{};
    if (space) sp = *space;
    std::vector<uint32_t> vpls, radices, lengths;
    const uint32_t vmask = sp.voices_per_lane_mask ? sp.voices_per_lane_mask : 3u;
    for (uint32_t v = 1; v <= 2; ++v)
        if (vmask & (1u << (v - 1))) vpls.push_back(v);
    const uint32_t rmask = sp.radix_mask ? sp.radix_mask : ((1u << 6) | (1u << 8) | (1u << 10));
    for (uint32_t r = 4; r <= 10; ++r)
        if (rmask & (1u << r)) radices.push_back(r);
    for (uint32_t bf : sp.block_frames)
        if (bf) lengths.push_back(bf);
    if (lengths.empty()) lengths.push_back(job->cfg.block_frames);
    if (vpls.empty() || radices.empty()) return fail(KC_ERR_INVALID, "empty tuning space");
    if ((vmask >> 2) || (rmask & ~0x7F0u)) return fail(KC_ERR_INVALID, "tuning mask names an unsupported value");
    const uint32_t preroll = sp.preroll_blocks ? sp.preroll_blocks : 16;
    const uint32_t timed = sp.timed_blocks ? sp.timed_blocks : 4;
    std::vector<ks_tune_result> all;
    for (uint32_t bf : lengths)
        if (int rc = tune_block_length(*job, bf, vpls, radices, preroll, timed, all)) return rc;
    size_t bi = 0;
    for (size_t i = 1; i < all.size(); ++i)
        if (all[i].voice_samples_per_s > all[bi].voice_samples_per_s) bi = i;
    *best = job->cfg;
    best->voices_per_lane = all[bi].voices_per_lane;
    best->sort_radix_bits = all[bi].sort_radix_bits;
    best->block_frames = all[bi].block_frames;
    if (results)
        for (size_t i = 0; i < all.size() && i < cap; ++i) results[i] = all[i];
    if (n) *n = (uint32_t)all.size();
    return KC_OK;
}

void ks_server_config_default(ks_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->mode = KS_MODE_BATCHED;
    c->device = 0;
    c->max_jobs = 256;
    c->host_threads = 0;
    c->vram_budget = 0;
    c->use_graph = 1;
    c->realtime_arrivals = 1;
    c->device_resample = 1;
}

uint64_t ks_hash_block(uint64_t h, const float* out, size_t n) {
    // FNV-1a over the block's 64-bit words (a trailing odd float on its own).
    if (h == 0) h = 0xcbf29ce484222325ull;
    const size_t words = n / 2;
    for (size_t i = 0; i < words; ++i) {
        uint64_t w;
        std::memcpy(&w, out + 2 * i, 8);
        h = (h ^ w) * 0x100000001b3ull;
    }
    if (n & 1) {
        uint32_t w;
        std::memcpy(&w, out + n - 1, 4);
        h = (h ^ w) * 0x100000001b3ull;
    }
    return h;
}

int ks_serve(const ks_server_config* cfg, const ks_job_spec* specs, uint32_t n_jobs, ks_job_result* results,
             ks_run_stats* stats) {
    if (!cfg || (n_jobs && (!specs || !results)) || !stats) return fail(KC_ERR_INVALID, "null argument");
    if (cfg->mode > KS_MODE_PARALLEL) return fail(KC_ERR_INVALID, "unknown server mode");
    if (cfg->max_jobs == 0 || cfg->max_jobs > 1024) return fail(KC_ERR_INVALID, "max_jobs must be in 1..=1024");
    std::memset(stats, 0, sizeof(*stats));
    if (n_jobs == 0) return KC_OK;
    // With autotune, every job runs with the tunables that won on the job
    // with the largest voice pool.
    std::vector<ks_job_spec> tuned;
    if (cfg->autotune) {
        uint32_t big = 0;
        for (uint32_t i = 1; i < n_jobs; ++i)
            if (specs[i].cfg.max_voices > specs[big].cfg.max_voices) big = i;
        ks_tune_space sp{};
        sp.preroll_blocks = 8;
        sp.timed_blocks = 3;
        kc_config best{};
        const auto t_tune = Clock::now();
        if (int rc = ks_autotune(&specs[big], &sp, &best, nullptr, 0, nullptr)) return rc;
        stats->tune_s = since(t_tune);
        stats->tuned_voices_per_lane = best.voices_per_lane;
        stats->tuned_sort_radix_bits = best.sort_radix_bits;
        tuned.assign(specs, specs + n_jobs);
        for (auto& t : tuned) {
            t.cfg.voices_per_lane = best.voices_per_lane;
            t.cfg.sort_radix_bits = best.sort_radix_bits;
        }
        specs = tuned.data();
    }
    std::vector<Job> jobs(n_jobs);
    std::vector<uint32_t> order(n_jobs);
    for (uint32_t i = 0; i < n_jobs; ++i) {
        jobs[i].id = i;
        jobs[i].spec = &specs[i];
        jobs[i].res = &results[i];
        std::memset(&results[i], 0, sizeof(results[i]));
        results[i].arrival_s = specs[i].arrival_s;
        order[i] = i;
        if (cfg->mode == KS_MODE_BATCHED && !same_batch_variant(specs[i].cfg, specs[0].cfg))
            return fail(KC_ERR_INVALID, "job " + std::to_string(i) +
                                            " differs from job 0 in device, block_frames, interpolation, "
                                            "strict_fp, mix_mode, voices_per_lane or sort_radix_bits");
        if (specs[i].cfg.device != cfg->device)
            return fail(KC_ERR_INVALID, "job " + std::to_string(i) + " is configured for another device");
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return specs[a].arrival_s < specs[b].arrival_s; });
    // Banks built during the run convert their samples on the server's GPU.
    int resample_device = (int)cfg->device;
    if (cfg->device_resample) kh_set_resampler(kc_resample_i16_batch, &resample_device);
    const auto t0 = Clock::now();
    const int rc = cfg->mode == KS_MODE_SEQUENTIAL ? serve_sequential(*cfg, jobs, order, *stats, t0)
                   : cfg->mode == KS_MODE_PARALLEL ? serve_parallel(*cfg, jobs, order, *stats, t0)
                                                   : serve_batched(*cfg, jobs, order, *stats, t0);
    if (cfg->device_resample) kh_set_resampler(nullptr, nullptr);
    stats->wall_s = since(t0);
    for (uint32_t i = 0; i < n_jobs; ++i) {
        stats->voice_samples += results[i].voice_samples;
        stats->job_blocks += results[i].blocks;
    }
    if (cfg->mode == KS_MODE_SEQUENTIAL) stats->host_threads = 1;
    return rc;
}

const char* ks_last_error(void) { return g_err.c_str(); }

}  // extern "C"
