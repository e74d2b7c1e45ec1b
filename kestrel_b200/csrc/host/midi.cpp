// midi.cpp -- the seeded synthetic event stream.
#include "midi.h"

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

SynthMidi::SynthMidi(const kh_midi_spec& s)
    : spec_(s), rng_(s.seed), offs_((uint64_t)std::max(1.0, 2.0 * (double)(s.ppq ? s.ppq : 9600) / 1000.0)) {
    if (spec_.ppq == 0) spec_.ppq = 9600;
    // 120 bpm: two quarter notes per second.
    ticks_per_s_ = 2.0 * (double)spec_.ppq;
    std::uniform_real_distribution<double> u(0.0, 1.0);
    phase_.resize(3 * std::max<uint32_t>(spec_.channels, 1));
    for (auto& p : phase_) p = u(rng_);
}

void SynthMidi::refill_onsets() {
    ons_.clear();
    on_pos_ = 0;
    const double window = 0.25;  // seconds of onsets generated at a time
    while (ons_.empty() && window_t_ < spec_.seconds && onsets_made_ < spec_.notes) {
        const double t0 = window_t_;
        const double t1 = std::min(spec_.seconds, t0 + window);
        window_t_ = t1;
        const double rate = (double)spec_.notes / std::max(spec_.seconds, 1e-9);
        const double share = std::clamp(spec_.cluster_share, 0.0, 1.0);
        const double mean_cluster = 0.5 * ((double)spec_.cluster_lo + (double)spec_.cluster_hi);
        std::vector<double> times;
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
        std::sort(times.begin(), times.end());
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
            ons_.push_back(o);
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

}  // namespace kh
