// midi.cpp -- the driver's event sources: the seeded synthetic stream and
// standard MIDI files.
#include "midi.h"

#include <cstdio>
#include <cstring>
#include <functional>

namespace kh {

void OffQueue::push(const Off& o) {
    const uint64_t b = o.tick / w_;
    ++size_;
    if (buckets_.empty()) base_ = b;
    if (b < base_) {
        // Earlier than every bucket held (only before the first pop reaches
        // it): open buckets down to it.
        buckets_.insert(buckets_.begin(), base_ - b, std::vector<Off>());
        base_ = b;
        pos_ = 0;
        front_sorted_ = false;
    }
    const uint64_t i = b - base_;
    if (i >= buckets_.size()) buckets_.resize(i + 1);
    std::vector<Off>& v = buckets_[i];
    if (i == 0 && front_sorted_) {
        // The bucket being consumed: keep its unconsumed part in order.
        v.insert(std::upper_bound(v.begin() + pos_, v.end(), o), o);
    } else {
        v.push_back(o);
    }
}

void OffQueue::settle() {
    while (pos_ >= buckets_.front().size()) {
        buckets_.pop_front();
        ++base_;
        pos_ = 0;
        front_sorted_ = false;
    }
    if (!front_sorted_) {
        std::sort(buckets_.front().begin(), buckets_.front().end());
        front_sorted_ = true;
    }
}

const OffQueue::Off& OffQueue::top() {
    settle();
    return buckets_.front()[pos_];
}

void OffQueue::pop() {
    settle();
    ++pos_;
    --size_;
    if (size_ == 0) {
        buckets_.clear();
        pos_ = 0;
        front_sorted_ = false;
    }
}

struct SynthMidi::WindowsAhead {
    static constexpr size_t DEPTH = 3;
    std::mutex m;
    std::condition_variable produced, consumed;
    std::deque<std::vector<On>> q;
    std::vector<std::vector<On>> spare;
    bool stop = false, ended = false;
    std::thread th;
};

SynthMidi::SynthMidi(const kh_midi_spec& s)
    : spec_(s), rng_(s.seed), offs_((uint64_t)std::max(1.0, 2.0 * (double)(s.ppq ? s.ppq : 9600) / 1000.0)) {
    if (spec_.ppq == 0) spec_.ppq = 9600;
    // 120 bpm: two quarter notes per second.
    ticks_per_s_ = 2.0 * (double)spec_.ppq;
    std::uniform_real_distribution<double> u(0.0, 1.0);
    phase_.resize(3 * std::max<uint32_t>(spec_.channels, 1));
    for (auto& p : phase_) p = u(rng_);
    const bool ctrl_draws = spec_.programs > 1 && spec_.program_period_s > 0.0;
    if (!ctrl_draws) {
        ahead_ = std::make_unique<WindowsAhead>();
        WindowsAhead* w = ahead_.get();
        w->th = std::thread([this, w] {
            for (;;) {
                std::vector<On> v;
                {
                    std::unique_lock<std::mutex> g(w->m);
                    w->consumed.wait(g, [w] { return w->stop || w->q.size() < WindowsAhead::DEPTH; });
                    if (w->stop) return;
                    if (!w->spare.empty()) {
                        v = std::move(w->spare.back());
                        w->spare.pop_back();
                    }
                }
                make_window(v);
                const bool last = v.empty();
                {
                    std::lock_guard<std::mutex> g(w->m);
                    w->q.push_back(std::move(v));
                }
                w->produced.notify_one();
                if (last) return;
            }
        });
    }
}

SynthMidi::~SynthMidi() {
    if (!ahead_) return;
    {
        std::lock_guard<std::mutex> g(ahead_->m);
        ahead_->stop = true;
    }
    ahead_->consumed.notify_all();
    ahead_->th.join();
}

// std::sort's result for a window's onset times, by a bucket sort: times
// lie in [lo, hi) (a cluster may run up to 1 ms past hi and lands in the
// last bucket), the bucket index is a monotone function of the time, and
// each bucket is sorted on its own. Any correct sort of the same values
// yields the same sequence.
static void sort_times(std::vector<double>& v, std::vector<double>& tmp, std::vector<uint32_t>& cnt, double lo,
                       double hi) {
    const size_t n = v.size();
    if (n < 64 || !(hi > lo)) {
        std::sort(v.begin(), v.end());
        return;
    }
    const size_t nb = n / 2;
    const double scale = (double)nb / (hi - lo);
    auto bucket = [&](double t) {
        const double x = (t - lo) * scale;
        const size_t i = x > 0.0 ? (size_t)x : 0;
        return i < nb ? i : nb - 1;
    };
    tmp.resize(n);
    cnt.assign(nb + 1, 0);
    for (size_t i = 0; i < n; ++i) ++cnt[bucket(v[i]) + 1];
    for (size_t b = 0; b < nb; ++b) cnt[b + 1] += cnt[b];
    for (size_t i = 0; i < n; ++i) tmp[cnt[bucket(v[i])]++] = v[i];
    size_t start = 0;  // cnt[b] is now the end of bucket b
    for (size_t b = 0; b < nb; ++b) {
        const size_t end = cnt[b];
        if (end - start > 16) {
            std::sort(tmp.begin() + (ptrdiff_t)start, tmp.begin() + (ptrdiff_t)end);
        } else {
            for (size_t i = start + 1; i < end; ++i) {
                const double x = tmp[i];
                size_t j = i;
                for (; j > start && tmp[j - 1] > x; --j) tmp[j] = tmp[j - 1];
                tmp[j] = x;
            }
        }
        start = end;
    }
    v.swap(tmp);
}

void SynthMidi::refill_onsets() {
    on_pos_ = 0;
    if (!ahead_) {
        make_window(ons_);
        return;
    }
    WindowsAhead* w = ahead_.get();
    std::unique_lock<std::mutex> g(w->m);
    if (w->ended) {
        ons_.clear();
        return;
    }
    if (ons_.capacity()) w->spare.push_back(std::move(ons_));
    w->produced.wait(g, [w] { return !w->q.empty(); });
    ons_ = std::move(w->q.front());
    w->q.pop_front();
    if (ons_.empty()) w->ended = true;
    g.unlock();
    w->consumed.notify_one();
}

// The next non-empty window's onsets in time order (empty at the end).
void SynthMidi::make_window(std::vector<On>& ons) {
    ons.clear();
    const double window = 0.25;  // seconds of onsets generated at a time
    while (ons.empty() && window_t_ < spec_.seconds && onsets_made_ < spec_.notes) {
        const double t0 = window_t_;
        const double t1 = std::min(spec_.seconds, t0 + window);
        window_t_ = t1;
        const double rate = (double)spec_.notes / std::max(spec_.seconds, 1e-9);
        const double share = std::clamp(spec_.cluster_share, 0.0, 1.0);
        const double mean_cluster = 0.5 * ((double)spec_.cluster_lo + (double)spec_.cluster_hi);
        std::vector<double>& times = times_;
        times.clear();
        std::poisson_distribution<uint64_t> bg((1.0 - share) * rate * (t1 - t0));
        std::uniform_real_distribution<double> ut(t0, t1);
        const uint64_t nbg = bg(rng_);
        for (uint64_t i = 0; i < nbg; ++i) times.push_back(ut(rng_));
        if (share > 0.0 && mean_cluster > 0.0) {
            std::poisson_distribution<uint64_t> nc(share * rate * (t1 - t0) / mean_cluster);
            std::uniform_int_distribution<uint32_t> csize(spec_.cluster_lo, std::max(spec_.cluster_lo, spec_.cluster_hi));
            const uint64_t k = nc(rng_);
            for (uint64_t c = 0; c < k; ++c) {
                const double start = ut(rng_);
                const uint32_t m = csize(rng_);
                std::uniform_real_distribution<double> uc(start, start + 0.001);
                for (uint32_t i = 0; i < m; ++i) times.push_back(uc(rng_));
            }
        }
        sort_times(times, times_tmp_, sort_cnt_, t0, t1);
        std::uniform_int_distribution<uint32_t> uch(0, std::max<uint32_t>(spec_.channels, 1) - 1);
        std::uniform_int_distribution<uint32_t> ukey(spec_.key_lo, std::max(spec_.key_lo, spec_.key_hi));
        std::uniform_int_distribution<uint32_t> uvel(std::max<uint32_t>(spec_.vel_lo, 1),
                                                     std::max(std::max<uint32_t>(spec_.vel_lo, 1), spec_.vel_hi));
        std::lognormal_distribution<double> dur(std::log(std::max(spec_.dur_median_s, 1e-6)), spec_.dur_sigma);
        for (double t : times) {
            if (onsets_made_ >= spec_.notes) break;
            On o;
            o.tick = tick_of(t);
            o.ch = (uint8_t)uch(rng_);
            o.key = (uint8_t)ukey(rng_);
            o.vel = (uint8_t)uvel(rng_);
            o.dur_s = dur(rng_);
            ons.push_back(o);
            ++onsets_made_;
        }
    }
}

// The controller schedule: at every step, per channel, a pitch bend and the
// CC7/CC11 curves (when cc_period_ms > 0), and every program_period_s a
// program change per channel. Step 0 sets each channel's first program.
bool SynthMidi::next_ctrl(uint64_t* tick, Event* ev, bool peek_only) {
    const uint32_t nch = std::max<uint32_t>(spec_.channels, 1);
    while (!ctrl_done_ && ctrl_sub_ >= ctrl_buf_.size()) {
        ctrl_buf_.clear();
        ctrl_sub_ = 0;
        const double period = spec_.cc_period_ms > 0.0 ? spec_.cc_period_ms * 1e-3 : 0.0;
        double t;
        if (ctrl_step_ == 0) {
            t = 0.0;
        } else if (period > 0.0) {
            t = (double)ctrl_step_ * period;
        } else if (spec_.program_period_s > 0.0) {
            t = (double)ctrl_step_ * spec_.program_period_s;
        } else {
            ctrl_done_ = true;
            break;
        }
        if (t >= spec_.seconds) {
            ctrl_done_ = true;
            break;
        }
        ctrl_tick_ = tick_of(t);
        const bool program_step =
            ctrl_step_ == 0 ||
            (spec_.program_period_s > 0.0 &&
             (period <= 0.0 ||
              (uint64_t)(t / spec_.program_period_s) != (uint64_t)((t - period) / spec_.program_period_s)));
        if (program_step && spec_.programs > 1) {
            std::uniform_int_distribution<uint32_t> up(0, spec_.programs - 1);
            for (uint32_t c = 0; c < nch; ++c) {
                Event e;
                e.type = EvType::Program;
                e.ch = (uint8_t)c;
                e.a = (uint8_t)(ctrl_step_ == 0 ? (c * spec_.programs / nch) % 128 : up(rng_) % 128);
                ctrl_buf_.push_back(e);
            }
        }
        if (period > 0.0) {
            for (uint32_t c = 0; c < nch; ++c) {
                const double w = 2.0 * M_PI;
                Event b;
                b.type = EvType::PitchBend;
                b.ch = (uint8_t)c;
                b.bend = (int16_t)std::lround(4096.0 * std::sin(w * (0.37 * t + phase_[3 * c])));
                ctrl_buf_.push_back(b);
                Event v;
                v.type = EvType::Cc;
                v.ch = (uint8_t)c;
                v.a = 7;
                v.b = (uint8_t)std::lround(100.0 + 27.0 * std::sin(w * (0.23 * t + phase_[3 * c + 1])));
                ctrl_buf_.push_back(v);
                Event x;
                x.type = EvType::Cc;
                x.ch = (uint8_t)c;
                x.a = 11;
                x.b = (uint8_t)std::lround(110.0 + 17.0 * std::sin(w * (0.61 * t + phase_[3 * c + 2])));
                ctrl_buf_.push_back(x);
            }
        }
        ++ctrl_step_;
    }
    if (ctrl_done_ && ctrl_sub_ >= ctrl_buf_.size()) return false;
    *tick = ctrl_tick_;
    if (!peek_only) *ev = ctrl_buf_[ctrl_sub_++];
    return true;
}

bool SynthMidi::next(uint64_t* tick, Event* ev) {
    if (on_pos_ >= ons_.size()) refill_onsets();
    const bool have_on = on_pos_ < ons_.size();
    const bool have_off = !offs_.empty();
    uint64_t ct = 0;
    Event dummy;
    const bool have_ctrl = next_ctrl(&ct, &dummy, true);
    if (!have_on && !have_off && !have_ctrl) return false;
    const uint64_t on_t = have_on ? ons_[on_pos_].tick : UINT64_MAX;
    const uint64_t off_t = have_off ? offs_.top().tick : UINT64_MAX;
    const uint64_t c_t = have_ctrl ? ct : UINT64_MAX;
    if (have_off && off_t <= c_t && off_t <= on_t) {
        const Off o = offs_.top();
        offs_.pop();
        *tick = o.tick;
        ev->type = EvType::NoteOff;
        ev->ch = o.ch;
        ev->a = o.key;
        ev->b = 0;
        return true;
    }
    if (have_ctrl && c_t <= on_t) {
        next_ctrl(tick, ev, false);
        return true;
    }
    const On o = ons_[on_pos_++];
    *tick = o.tick;
    ev->type = EvType::NoteOn;
    ev->ch = o.ch;
    ev->a = o.key;
    ev->b = o.vel;
    uint64_t off = tick_of((double)o.tick / ticks_per_s_ + o.dur_s);
    if (off <= o.tick) off = o.tick + 1;
    offs_.push(Off{off, off_seq_++, o.ch, o.key});  // (tick, seq) order, as pops return them
    return true;
}

AheadSource::AheadSource(std::unique_ptr<EventSource> inner, size_t chunk, size_t depth)
    : inner_(std::move(inner)), div_(inner_->division()), chunk_(std::max<size_t>(chunk, 1)),
      depth_(std::max<size_t>(depth, 1)) {
    th_ = std::thread([this] { run(); });
}

AheadSource::~AheadSource() {
    {
        std::lock_guard<std::mutex> g(m_);
        stop_ = true;
    }
    consumed_.notify_all();
    th_.join();
}

void AheadSource::run() {
    for (;;) {
        Chunk c;
        {
            std::unique_lock<std::mutex> g(m_);
            consumed_.wait(g, [this] { return stop_ || q_.size() < depth_; });
            if (stop_) return;
            if (!spare_.empty()) {
                c = std::move(spare_.back());
                spare_.pop_back();
            }
        }
        c.ticks.clear();
        c.evs.clear();
        c.last = false;
        uint64_t tick;
        Event ev;
        while (c.evs.size() < chunk_) {
            if (!inner_->next(&tick, &ev)) {
                c.last = true;
                break;
            }
            c.ticks.push_back(tick);
            c.evs.push_back(ev);
        }
        const bool last = c.last;
        {
            std::lock_guard<std::mutex> g(m_);
            q_.push_back(std::move(c));
        }
        produced_.notify_one();
        if (last) return;
    }
}

bool AheadSource::next(uint64_t* tick, Event* ev) {
    while (pos_ >= cur_.evs.size()) {
        if (ended_ || cur_.last) {
            ended_ = true;
            return false;
        }
        std::unique_lock<std::mutex> g(m_);
        if (!cur_.evs.empty() || cur_.ticks.capacity()) spare_.push_back(std::move(cur_));
        produced_.wait(g, [this] { return !q_.empty(); });
        cur_ = std::move(q_.front());
        q_.pop_front();
        pos_ = 0;
        g.unlock();
        consumed_.notify_one();
    }
    *tick = cur_.ticks[pos_];
    *ev = cur_.evs[pos_];
    ++pos_;
    return true;
}

}  // namespace kh

// ---- standard MIDI files ---------------------------------------------------------

namespace kh {

namespace {
constexpr size_t TRACK_BUF = 256 * 1024;

uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }
uint16_t be16(const uint8_t* p) { return (uint16_t)(p[0] << 8 | p[1]); }
}  // namespace

// TrackReader (src/midi.rs:39-236): one track chunk with its own file handle
// and read window; decodes one event at a time, keeping running status.
struct SmfStream::Track {
    std::FILE* f = nullptr;
    std::vector<uint8_t> buf;
    size_t pos = 0, filled = 0;
    uint64_t remaining = 0;
    uint64_t tick = 0;
    uint8_t running = 0;
    bool ended = false;

    ~Track() {
        if (f) std::fclose(f);
    }
    bool fill() {
        if (remaining == 0) return false;
        const size_t want = (size_t)std::min<uint64_t>(remaining, TRACK_BUF);
        const size_t got = std::fread(buf.data(), 1, want, f);
        remaining -= got;
        pos = 0;
        filled = got;
        return got > 0;
    }
    bool byte(uint8_t* b) {
        if (pos == filled && !fill()) return false;
        *b = buf[pos++];
        return true;
    }
    bool varlen(uint64_t* v) {
        *v = 0;
        for (int i = 0; i < 8; ++i) {
            uint8_t b;
            if (!byte(&b)) return false;
            *v = (*v << 7) | (uint64_t)(b & 0x7F);
            if (!(b & 0x80)) return true;
        }
        return false;
    }
    bool skip(uint64_t n) {
        while (n > 0) {
            if (pos == filled && !fill()) return false;
            const uint64_t take = std::min<uint64_t>(filled - pos, n);
            pos += (size_t)take;
            n -= take;
        }
        return true;
    }
    // TrackReader::next_event (src/midi.rs:126-236). False at the end of the
    // track, or where it stops making sense.
    bool next_event(Event* ev) {
        if (ended) return false;
        auto end = [&] {
            ended = true;
            return false;
        };
        uint64_t delta;
        if (!varlen(&delta)) return end();
        tick += delta;
        uint8_t status;
        if (!byte(&status)) return end();
        uint8_t first = 0;
        if (status < 0x80) {
            // Running status: the byte is the first data byte of a message
            // with the previous channel status.
            first = status;
            status = running;
            if (status < 0x80) return end();  // data before any status byte
        } else {
            if (status < 0xF0) running = status;
            else if (status == 0xFF) running = 0;  // only meta clears it
            if (status != 0xFF && status != 0xF0 && status != 0xF7 && !byte(&first)) return end();
        }
        const uint8_t ch = status & 0x0F;
        *ev = Event{};
        ev->ch = ch;
        uint8_t b2;
        switch (status & 0xF0) {
            case 0x80:
                if (!byte(&b2)) return false;
                ev->type = EvType::NoteOff;
                ev->a = first & 0x7F;
                return true;
            case 0x90:
                if (!byte(&b2)) return false;
                ev->a = first & 0x7F;
                if (b2 == 0) {
                    ev->type = EvType::NoteOff;
                } else {
                    ev->type = EvType::NoteOn;
                    ev->b = b2 & 0x7F;
                }
                return true;
            case 0xA0:
                if (!byte(&b2)) return false;
                ev->type = EvType::Other;
                return true;
            case 0xB0:
                if (!byte(&b2)) return false;
                ev->type = EvType::Cc;
                ev->a = first & 0x7F;
                ev->b = b2 & 0x7F;
                return true;
            case 0xC0:
                ev->type = EvType::Program;
                ev->a = first & 0x7F;
                return true;
            case 0xD0:
                ev->type = EvType::Other;
                return true;
            case 0xE0: {
                if (!byte(&b2)) return false;
                const int16_t raw = (int16_t)(((int16_t)(b2 & 0x7F) << 7) | (int16_t)(first & 0x7F));
                ev->type = EvType::PitchBend;
                ev->bend = (int16_t)(raw - 8192);
                return true;
            }
            default:
                break;
        }
        ev->type = EvType::Other;
        ev->ch = 0;
        if (status == 0xFF) {
            uint8_t meta;
            uint64_t len;
            if (!byte(&meta) || !varlen(&len)) return false;
            if (meta == 0x2F) {
                if (!skip(len)) return false;
                ended = true;
                return true;
            }
            if (meta == 0x51 && len == 3) {
                uint8_t a, b, c;
                if (!byte(&a) || !byte(&b) || !byte(&c)) return false;
                ev->type = EvType::Tempo;
                ev->tempo = (uint32_t)a << 16 | (uint32_t)b << 8 | c;
                return true;
            }
            return skip(len);
        }
        if (status == 0xF0 || status == 0xF7) {
            uint64_t len;
            if (!varlen(&len)) return false;
            return skip(len);
        }
        return true;  // other system messages carry no data here
    }
};

SmfStream::~SmfStream() = default;

// MidiStream::open (src/midi.rs:259-363).
std::unique_ptr<SmfStream> SmfStream::open(const std::string& path, std::string* err) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        *err = "opening " + path;
        return nullptr;
    }
    std::fseek(f, 0, SEEK_END);
    const uint64_t file_len = (uint64_t)std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    uint8_t hdr[14];
    if (std::fread(hdr, 1, 14, f) != 14) {
        std::fclose(f);
        *err = path + ": too short for an SMF header";
        return nullptr;
    }
    if (std::memcmp(hdr, "MThd", 4) != 0) {
        std::fclose(f);
        *err = path + ": not a standard MIDI file";
        return nullptr;
    }
    std::unique_ptr<SmfStream> s(new SmfStream());
    const uint64_t hdr_len = be32(hdr + 4);
    s->format_ = be16(hdr + 8);
    const int16_t div_raw = (int16_t)be16(hdr + 12);
    if (div_raw > 0) {
        s->division_.ppq = (uint32_t)div_raw;
    } else {
        s->division_.smpte = true;
        s->division_.fps = (uint8_t)(-(div_raw >> 8));
        s->division_.ticks_per_frame = (uint8_t)(div_raw & 0xFF);
    }
    // Walk the chunk headers; a zero-length unknown chunk is trailing padding
    // (exporters pad with zeros), where the walk stops.
    std::vector<std::pair<uint64_t, uint64_t>> locs;
    uint64_t offset = 8 + hdr_len;
    while (offset + 8 <= file_len) {
        uint8_t ch[8];
        if (std::fseek(f, (long)offset, SEEK_SET) != 0 || std::fread(ch, 1, 8, f) != 8) break;
        const uint64_t data_start = offset + 8;
        const uint64_t len = std::min<uint64_t>(be32(ch + 4), file_len > data_start ? file_len - data_start : 0);
        if (std::memcmp(ch, "MTrk", 4) == 0) locs.emplace_back(data_start, len);
        else if (len == 0) break;
        offset = data_start + len;
    }
    std::fclose(f);
    if (locs.empty()) {
        *err = path + ": no MTrk chunks";
        return nullptr;
    }
    for (const auto& [off, len] : locs) {
        auto t = std::make_unique<Track>();
        t->f = std::fopen(path.c_str(), "rb");
        if (!t->f || std::fseek(t->f, (long)off, SEEK_SET) != 0) {
            *err = "opening " + path;
            return nullptr;
        }
        t->buf.resize(TRACK_BUF);
        t->remaining = len;
        s->readers_.push_back(std::move(t));
    }
    s->pending_.resize(s->readers_.size());
    for (uint32_t i = 0; i < s->readers_.size(); ++i)
        if (s->readers_[i]->next_event(&s->pending_[i])) s->heap_.emplace_back(s->readers_[i]->tick, i);
    std::make_heap(s->heap_.begin(), s->heap_.end(), std::greater<>());
    return s;
}

// MidiStream::next (src/midi.rs:365-374): the smallest (tick, track) first.
bool SmfStream::next(uint64_t* tick, Event* ev) {
    if (heap_.empty()) return false;
    std::pop_heap(heap_.begin(), heap_.end(), std::greater<>());
    const auto [t, i] = heap_.back();
    heap_.pop_back();
    *tick = t;
    *ev = pending_[i];
    if (readers_[i]->next_event(&pending_[i])) {
        heap_.emplace_back(readers_[i]->tick, i);
        std::push_heap(heap_.begin(), heap_.end(), std::greater<>());
    }
    return true;
}

}  // namespace kh
