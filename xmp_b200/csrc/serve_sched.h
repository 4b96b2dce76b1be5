// Host-side bookkeeping of the modexp serving loop: the per-precision slot
// ring that bounds device memory (admission control) and the rule that
// decides when pending requests become a launch wave.  No CUDA types, so the
// same header is unit-tested on a CPU-only machine.
#pragma once
#include <cstdint>

namespace xmpb {
namespace serve {

// Ring of op slots in device memory.  A wave takes a contiguous range of
// slots rounded up to `granule`; a range never wraps (the unused tail is
// taken along with it).  Ranges are released oldest first.
class SlotRing {
 public:
  SlotRing() = default;
  SlotRing(uint32_t capacity, uint32_t granule) : cap_(capacity / granule * granule), gran_(granule) {}

  uint32_t capacity() const { return cap_; }
  uint32_t used() const { return used_; }
  uint32_t granule() const { return gran_; }

  // Largest op count a single wave can take right now.
  uint32_t largest_free() const {
    uint32_t free_total = cap_ - used_;
    uint32_t run = cap_ - head_;  // head to the end of the ring
    if (run >= free_total) return free_total;
    // the free space is [head, cap) plus [0, free_total - run)
    uint32_t wrap = free_total - run;
    return run > wrap ? run : wrap;
  }

  // Reserves slots for n ops.  On success *first is the first slot and
  // *taken the ring space consumed (to hand back to release()).
  bool alloc(uint32_t n, uint32_t *first, uint32_t *taken) {
    if (n == 0 || gran_ == 0) return false;
    uint64_t r = ((uint64_t)n + gran_ - 1) / gran_ * gran_;
    if (r > cap_) return false;
    uint32_t free_total = cap_ - used_;
    uint32_t run = cap_ - head_;
    if (r <= run && r <= free_total) {
      *first = head_;
      *taken = (uint32_t)r;
      head_ = (head_ + (uint32_t)r) % cap_;
      used_ += (uint32_t)r;
      return true;
    }
    // skip the tail [head, cap) and start again at slot 0
    if (run < free_total && r <= free_total - run) {
      *first = 0;
      *taken = run + (uint32_t)r;
      head_ = (uint32_t)r % cap_;
      used_ += *taken;
      return true;
    }
    return false;
  }

  void release(uint32_t taken) {
    used_ = taken > used_ ? 0 : used_ - taken;
    if (used_ == 0) head_ = 0;  // nothing outstanding: restart at slot 0
  }

 private:
  uint32_t cap_ = 0, gran_ = 1, head_ = 0, used_ = 0;
};

// When to turn pending requests into a wave: as soon as a launch stream is
// idle.  A wave put behind another one on a busy stream would wait for all of
// it, so while every stream is busy requests stay pending and merge into one
// larger wave when a stream frees up -- batches grow with the load by
// themselves.  A full wave (max_wave_ops) is the only other trigger.
struct WavePolicy {
  uint32_t max_wave_ops = 4096;

  bool should_launch(uint32_t pending_ops, uint32_t idle_streams) const {
    if (pending_ops == 0) return false;
    return idle_streams > 0;
  }
};

}  // namespace serve
}  // namespace xmpb
