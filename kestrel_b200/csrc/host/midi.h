// midi.h -- events, the tempo clock (src/midi.rs:17-34, 376-431), and the
// seeded synthetic event stream that stands in for a black-MIDI file.
#pragma once

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <random>
#include <thread>
#include <vector>

#include "../../../include/kestrel_host.h"

namespace kh {

// midi::Event (src/midi.rs:17-29).
enum class EvType : uint8_t { NoteOn, NoteOff, Cc, Program, PitchBend, Tempo, Other };

struct Event {
    EvType type = EvType::Other;
    uint8_t ch = 0, a = 0, b = 0;  // NoteOn: key, vel; NoteOff: key; Cc: num, val; Program: val
    int16_t bend = 0;              // PitchBend value, -8192..8191
    uint32_t tempo = 0;            // microseconds per quarter note
};

// midi::Division (src/midi.rs:31-37).
struct Division {
    bool smpte = false;
    uint32_t ppq = 960;
    uint8_t fps = 0, ticks_per_frame = 0;
};

// TempoClock (src/midi.rs:378-431): ticks to output frames, following tempo
// changes as they arrive in the merged stream. SMPTE division ignores tempo.
struct TempoClock {
    Division division;
    double sample_rate = 48000.0;
    uint64_t base_tick = 0;
    double base_frame = 0.0;
    double frames_per_tick = 0.0;

    TempoClock() = default;
    TempoClock(Division d, uint32_t rate) : division(d), sample_rate((double)rate) { set_tempo_raw(500000); }
    void set_tempo_raw(uint32_t us_per_qn) {
        if (division.smpte) {
            const double tps = (double)std::max<uint8_t>(division.fps, 1) *
                               (double)std::max<uint8_t>(division.ticks_per_frame, 1);
            frames_per_tick = sample_rate / tps;
        } else {
            const double p = (double)std::max<uint32_t>(division.ppq, 1);
            frames_per_tick = ((double)us_per_qn * 1e-6) * sample_rate / p;
        }
    }
    void set_tempo(uint64_t tick, uint32_t us_per_qn) {
        if (division.smpte) return;
        base_frame = frame_at(tick);
        base_tick = tick;
        set_tempo_raw(us_per_qn);
    }
    double frame_at(uint64_t tick) const { return base_frame + (double)(tick - base_tick) * frames_per_tick; }
};

// Where the driver's events come from: a MIDI file or the synthetic stream.
class EventSource {
   public:
    virtual ~EventSource() = default;
    // Next event in tick order; false when the stream is exhausted.
    virtual bool next(uint64_t* tick, Event* ev) = 0;
    virtual Division division() const = 0;
};

// Another source run on its own thread, up to `depth` chunks of `chunk`
// events ahead of the reader. The events and their order are the inner
// source's; only the thread that produces them differs, so the driver's
// input blocks are unchanged while generating or parsing events overlaps
// the driver's own work.
class AheadSource : public EventSource {
   public:
    AheadSource(std::unique_ptr<EventSource> inner, size_t chunk = 8192, size_t depth = 64);
    ~AheadSource() override;
    bool next(uint64_t* tick, Event* ev) override;
    Division division() const override { return div_; }

   private:
    struct Chunk {
        std::vector<uint64_t> ticks;
        std::vector<Event> evs;
        bool last = false;  // the inner source is exhausted after this chunk
    };
    void run();

    std::unique_ptr<EventSource> inner_;
    Division div_;
    size_t chunk_, depth_;
    std::mutex m_;
    std::condition_variable produced_, consumed_;
    std::deque<Chunk> q_;
    std::vector<Chunk> spare_;  // consumed chunks handed back for reuse
    bool stop_ = false;
    Chunk cur_;
    size_t pos_ = 0;
    bool ended_ = false;
    std::thread th_;
};

// MidiStream (src/midi.rs:239-374): a standard MIDI file read a window at a
// time per track (256 KiB each, so a 40 GB file costs the memory of a small
// one) and merged into one tick-ordered stream, ties broken by track index.
class SmfStream : public EventSource {
   public:
    // Returns null (with `err` set) when the file is not a usable SMF.
    static std::unique_ptr<SmfStream> open(const std::string& path, std::string* err);
    ~SmfStream() override;
    bool next(uint64_t* tick, Event* ev) override;
    Division division() const override { return division_; }
    uint16_t format() const { return format_; }
    uint16_t tracks() const { return (uint16_t)readers_.size(); }

   private:
    struct Track;
    SmfStream() = default;
    std::vector<std::unique_ptr<Track>> readers_;
    std::vector<Event> pending_;
    std::vector<std::pair<uint64_t, uint32_t>> heap_;  // min-heap of (tick, track)
    Division division_;
    uint16_t format_ = 0;
};

// Pending note-offs, popped in (tick, seq) order. A calendar queue: one
// unsorted bucket per BUCKET ticks, and the bucket being consumed sorted once
// when it is reached. Pushes append (an off landing in the bucket being
// consumed is inserted in order), so a stream holding millions of pending
// offs costs a sort of each ~1 ms bucket instead of a heap operation with a
// cache miss per level for every note.
class OffQueue {
   public:
    struct Off {
        uint64_t tick, seq;
        uint8_t ch, key;
        bool operator<(const Off& o) const { return tick != o.tick ? tick < o.tick : seq < o.seq; }
    };
    explicit OffQueue(uint64_t bucket_ticks) : w_(bucket_ticks ? bucket_ticks : 1) {}
    bool empty() const { return size_ == 0; }
    void push(const Off& o);
    // The smallest pending off; only when !empty().
    const Off& top();
    void pop();

   private:
    void settle();  // make buckets_.front() the first non-empty bucket, sorted
    uint64_t w_;
    std::deque<std::vector<Off>> buckets_;  // bucket base_ + i
    uint64_t base_ = 0;
    size_t pos_ = 0;                        // consumed prefix of buckets_.front()
    bool front_sorted_ = false;
    size_t size_ = 0;
};

// The synthetic stream. Onsets are generated one window of time at a time:
// background notes as a Poisson process, plus (optionally) 1 ms clusters of
// many simultaneous notes; every onset schedules its note-off in an OffQueue.
// Controller curves and program changes run on their own schedule. The three
// sources are merged by tick (at equal ticks: offs, then controllers, then
// ons), so the stream is a pure function of the spec.
class SynthMidi : public EventSource {
   public:
    explicit SynthMidi(const kh_midi_spec& s);
    ~SynthMidi() override;
    // Next event in tick order; false when the stream is exhausted.
    bool next(uint64_t* tick, Event* ev) override;
    Division division() const override {
        Division d;
        d.ppq = spec_.ppq;
        return d;
    }

   private:
    using Off = OffQueue::Off;
    struct On {
        uint64_t tick;
        uint8_t ch, key, vel;
        double dur_s;
    };
    void refill_onsets();
    void make_window(std::vector<On>& out);
    bool next_ctrl(uint64_t* tick, Event* ev, bool peek_only);
    uint64_t tick_of(double t) const { return (uint64_t)std::llround(t * ticks_per_s_); }

    kh_midi_spec spec_;
    std::mt19937_64 rng_;
    double ticks_per_s_;
    double window_t_ = 0.0;             // onsets generated up to here
    uint64_t onsets_made_ = 0;
    std::vector<On> ons_;
    size_t on_pos_ = 0;
    OffQueue offs_;
    uint64_t off_seq_ = 0;
    // controller schedule
    uint64_t ctrl_step_ = 0;            // index of the next controller time step
    uint32_t ctrl_sub_ = 0;             // which event within the step
    std::vector<Event> ctrl_buf_;
    uint64_t ctrl_tick_ = 0;
    bool ctrl_done_ = false;
    std::vector<double> phase_;         // per-channel curve phases
    std::vector<double> times_, times_tmp_;
    std::vector<uint32_t> sort_cnt_;
    // Onset windows made on a thread of their own, when the controller
    // schedule never draws from rng_ (no program changes after the first):
    // then the draws are the windows' alone and their order cannot depend
    // on how windows and controller events interleave.
    struct WindowsAhead;
    std::unique_ptr<WindowsAhead> ahead_;
};

}  // namespace kh
