// Host structural walk over a pool image: the counterpart of the reference's
// validate_tree_structure (include/gpu_blink_tree.hpp:742-900,
// include/gpu_versioned_blink_tree.hpp:1098-1259). It resolves every node to the version visible
// at the requested snapshot and checks, level by level from the root: key order inside nodes,
// that every key lies in [low fence, high key), levels, right links (the last node of a level has
// high key 0xFFFFFFFF and no sibling), that no node is left locked, and that every node of a level
// is referenced by exactly one entry of the level above, and that each node's stored low fence
// equals the high key of its left neighbour. Unlike the reference it needs no
// allocator bookkeeping, so it works for every pool layout.
#include <algorithm>
#include <iterator>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mvbt.h"

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kNone  = 0x0FFFFFFFu;
constexpr uint32_t kMask  = 0x0FFFFFFFu;
constexpr uint32_t kLock  = 0x80000000u;
constexpr int kData       = 13;

struct host_node {
  const uint32_t* w;
  uint32_t key(int p) const { return w[2 * p]; }
  uint32_t val(int p) const { return w[2 * p + 1]; }
  uint32_t low() const { return w[26]; }
  uint32_t high() const { return w[28]; }
  uint32_t mod() const { return w[27]; }  // bit31 lock | modification count
  uint32_t ts() const { return w[30]; }
  uint32_t level() const { return w[31] >> 28; }
  uint32_t older() const { return w[31] & kMask; }
  uint32_t sibling() const { return w[29] & kMask; }
};

}  // namespace

extern "C" int mvbt_validate_image_detail(const uint32_t* img, uint64_t nn, int versioned,
                                          uint32_t ts, mvbt_report* rep, char* detail,
                                          uint64_t detail_len) {
  if (!img || !rep || nn == 0) return MVBT_ERR_BAD_ARG;
  std::string log;
  auto note = [&](const char* what, int level, uint32_t slot, uint32_t a, uint32_t b) {
    if (log.size() > 4000) return;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "%s level=%d slot=%u a=%u b=%u; ", what, level, slot, a, b);
    log += buf;
  };
  std::memset(rep, 0, sizeof(*rep));
  rep->nodes_allocated = nn;
  const bool snap      = versioned && ts != 0xFFFFFFFFu;
  auto node            = [&](uint32_t i) { return host_node{img + (size_t)i * 32}; };
  uint32_t violations  = 0;
  auto resolve         = [&](uint32_t i) -> uint32_t {
    uint64_t hops = 0;
    while (snap && i < nn && node(i).ts() > ts) {
      i = node(i).older();
      if (++hops > nn) return kNone;
    }
    return i < nn ? i : kNone;
  };
  uint32_t root = resolve(0);
  if (root == kNone) {
    rep->violations = 1;
    return MVBT_ERR_CORRUPT;
  }
  const int top  = (int)node(root).level();  // node 0 is the anchor, one level above the top
  rep->height    = (uint32_t)top;
  uint32_t first = 0;  // slot index of the leftmost node of the level
  std::vector<uint32_t> child_slots;
  for (int level = top; level >= 0; --level) {
    std::vector<uint32_t> slots, next_children;
    uint32_t slot = first, low = 0;
    uint64_t guard = 0;
    while (slot != kNone) {
      if (++guard > nn + 1) {
        ++violations;
        note("sibling-cycle", level, slot, 0, 0);
        break;
      }
      uint32_t v = resolve(slot);
      if (v == kNone) {
        ++violations;
        note("no-version", level, slot, 0, 0);
        break;
      }
      host_node x = node(v);
      slots.push_back(slot);
      if ((int)x.level() != level) {
        ++violations;
        note("level", level, slot, x.level(), 0);
      }
      if (x.low() != low) {
        ++violations;
        note("stored-low-fence", level, slot, x.low(), low);
      }
      if (x.mod() & kLock) ++rep->locked_nodes;
      uint32_t prev = 0;
      bool have     = false;
      int cnt       = 0;
      for (int p = 0; p < kData; ++p) {
        uint32_t k = x.key(p);
        if (k == kEmpty) {
          for (int q = p; q < kData; ++q)
            if (x.key(q) != kEmpty) {  // valid pairs form a prefix
              ++violations;
              note("hole", level, slot, (uint32_t)q, x.key(q));
            }
          break;
        }
        ++cnt;
        if (have && k <= prev) {
          ++violations;
          note("order", level, slot, prev, k);
        }
        if (k < low || k >= x.high()) {
          ++violations;
          note(k < low ? "below-fence" : "above-high", level, slot, k, k < low ? low : x.high());
        }
        prev = k;
        have = true;
        if (level == 0) {
          ++rep->keys;
          rep->key_checksum += (uint64_t)k * 0x9E3779B1ull + x.val(p);
        } else {
          next_children.push_back(x.val(p));
        }
      }
      if (level > 0 && cnt == 0) {
        ++violations;
        note("empty-interior", level, slot, 0, 0);
      }
      if (level == 0) ++rep->leaves;
      else ++rep->interior;
      if (x.high() <= low && x.high() != kEmpty) {
        ++violations;
        note("fence-order", level, slot, low, x.high());
      }
      low  = x.high();
      slot = x.sibling();
      if (slot == kNone && x.high() != kEmpty) {
        ++violations;
        note("chain-end", level, v, x.high(), 0);
      }
    }
    if (level < top) {
      std::vector<uint32_t> a = slots, b = child_slots;
      std::sort(a.begin(), a.end());
      std::sort(b.begin(), b.end());
      if (a != b) {
        ++violations;
        std::vector<uint32_t> miss, extra;
        std::set_difference(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(miss));
        std::set_difference(b.begin(), b.end(), a.begin(), a.end(), std::back_inserter(extra));
        note("parent-links", level, miss.empty() ? 0 : miss[0], (uint32_t)miss.size(),
             (uint32_t)extra.size());
        for (size_t i = 0; i < miss.size() && i < 4; ++i) note("  unposted", level, miss[i], 0, 0);
        for (size_t i = 0; i < extra.size() && i < 4; ++i) note("  dangling", level, extra[i], 0, 0);
      }
    }
    child_slots = next_children;
    if (level > 0) {
      uint32_t v = resolve(first);
      if (v == kNone) break;
      first = node(v).val(0);
    }
  }
  if (rep->interior) --rep->interior;  // the anchor is not a tree node
  rep->violations = violations;
  if (detail && detail_len) {
    size_t c = std::min<size_t>(log.size(), detail_len - 1);
    std::memcpy(detail, log.data(), c);
    detail[c] = 0;
  }
  return violations ? MVBT_ERR_CORRUPT : MVBT_OK;
}

extern "C" int mvbt_validate_image(const uint32_t* img, uint64_t nn, int versioned, uint32_t ts,
                                   mvbt_report* rep) {
  return mvbt_validate_image_detail(img, nn, versioned, ts, rep, nullptr, 0);
}
