// Result rows of the daemon: member expansion of deduplicated layers, the self-join row rules and the frame
// encoding of the wire protocol. The rules follow op_join / op_relate / op_dwithin / op_cluster of
// daemon/gpujoind.cu (lines cited per function); the encoding follows daemon/protocol.h.
#pragma once
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/gsp_protocol.h"

namespace gsjd {

// Input-row ids of a layer, packed (one buffer + offsets).
struct IdTable {
  std::string buf;
  std::vector<uint64_t> off{0};
  void add(const char* p, size_t n) { buf.append(p, n); off.push_back(buf.size()); }
  size_t size() const { return off.size() - 1; }
  const char* data(size_t i) const { return buf.data() + off[i]; }
  size_t len(size_t i) const { return off[i + 1] - off[i]; }
};

// Rows a distinct geometry stands for (Layer::members, gpujoind.cu:71-74). moff == nullptr: not deduplicated.
struct Members {
  const uint64_t* moff = nullptr;
  const uint32_t* midx = nullptr;
  uint64_t count(uint32_t g) const { return moff ? moff[g + 1] - moff[g] : 1; }
  template <class F> void each(uint32_t g, F&& f) const {
    if (!moff) { f(g); return; }
    for (uint64_t k = moff[g]; k < moff[g + 1]; k++) f(midx[k]);
  }
};

// The rows of one engine pair (a, b): out(ra, rb, transposed). Self-joins get each unordered pair once from the
// engine; "all" mirrors it, "distinct" keeps lo < hi (gpujoind.cu:271-283, 356-367, 471-481).
template <class F>
inline void pair_rows(uint32_t a, uint32_t b, const Members& A, const Members& B, bool same, bool distinct, F&& out) {
  const bool diag = same && a == b;
  A.each(a, [&](uint32_t ra) {
    B.each(b, [&](uint32_t rb) {
      if (!same) { out(ra, rb, false); return; }
      if (distinct) {
        if (ra == rb || (diag && ra > rb)) return;
        if (ra < rb) out(ra, rb, false);
        else out(rb, ra, !diag);
        return;
      }
      out(ra, rb, false);
      if (!diag) out(rb, ra, true);
    });
  });
}

// Row count of one pair without expanding it (stats-only requests, gpujoind.cu:257-267).
inline uint64_t pair_row_count(uint32_t a, uint32_t b, const Members& A, const Members& B, bool same, bool distinct) {
  const uint64_t ma = A.count(a), mb = B.count(b);
  if (!same) return ma * mb;
  if (a == b) return distinct ? ma * (ma - 1) / 2 : ma * ma;
  return distinct ? ma * mb : 2 * ma * mb;
}

// Frames of rows: { u32 nrows, rows } closed once they hold GSP_FRAME_BYTES (FrameBuf, gpujoind.cu:178-190).
// A raw grow-only buffer: one capacity check and one copy per field; reset() keeps the capacity for the next
// request.
class FrameWriter {
 public:
  uint64_t rows = 0;
  const char* data() const { return buf_.get(); }
  size_t size() const { return len_; }
  void reset() { len_ = 0; rows = 0; fstart_ = 0; cnt_ = 0; }
  void reserve(size_t n) { if (n > cap_) grow(n); }
  void begin() { fstart_ = len_; ensure(4); len_ += 4; cnt_ = 0; }
  void id(const char* p, size_t n) {
    const uint16_t l = (uint16_t)(n < 65535 ? n : 65535);
    ensure(2 + (size_t)l);
    std::memcpy(buf_.get() + len_, &l, 2);
    std::memcpy(buf_.get() + len_ + 2, p, l);
    len_ += 2 + (size_t)l;
  }
  void f64(double x) { put(&x, 8); }
  void u32(uint32_t x) { put(&x, 4); }
  void raw(const char* p, size_t n) { put(p, n); }
  void row_done() {
    cnt_++; rows++;
    if (len_ - fstart_ >= GSP_FRAME_BYTES) { close(); begin(); }
  }
  void finish() { if (cnt_) close(); else len_ = fstart_; }

 private:
  void put(const void* p, size_t n) { ensure(n); std::memcpy(buf_.get() + len_, p, n); len_ += n; }
  void ensure(size_t n) { if (len_ + n > cap_) grow(len_ + n); }
  void grow(size_t need) {
    const size_t c = std::max(need, 2 * cap_ + 4096);
    std::unique_ptr<char[]> b(new char[c]);
    if (len_) std::memcpy(b.get(), buf_.get(), len_);
    buf_ = std::move(b);
    cap_ = c;
  }
  void close() { std::memcpy(buf_.get() + fstart_, &cnt_, 4); }
  std::unique_ptr<char[]> buf_;
  size_t len_ = 0, cap_ = 0, fstart_ = 0;
  uint32_t cnt_ = 0;
};

}  // namespace gsjd
