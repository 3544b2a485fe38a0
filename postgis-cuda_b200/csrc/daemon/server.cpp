// gsjd: serves resident layers over the gpujoind wire protocol (gsp_protocol.h) with the gsj engine.
//
// Behaviour follows daemon/gpujoind.cu of landstats-us/postgis-cuda: the same ops, argument checks, row rules,
// frame format and stats keys, so its Postgres extension works unchanged. Differences, by design:
//  - layers come from files (binary COPY / .gset / .pset, resolved inside --data-dir) instead of SQL over libpq;
//    LOAD_QUERY and LOAD's row filter need PostgreSQL and answer with an error;
//  - GPU work runs on pools of engine contexts (--workers, each its own CUDA stream and scratch) sharing the
//    resident layers, so requests that arrive while others run are admitted and overlap on the GPU instead of
//    queueing behind one device lock (g_gpu, gpujoind.cu:35). Small requests use high-priority streams. Admission
//    is first come, first served per pool, as a context and the request's scratch-memory estimate (within
//    --mem-budget-gb) become free.
//  - optionally, rows stream while the GPU works: with --stream-batch N, JOIN, RELATE and DWITHIN run in probe
//    batches of N query geometries and each batch's rows are encoded and written by a sender thread while the
//    engine refines the next batch. The default (0) is the reference's scheme: one batch, rows sent after it.
//  - rows are encoded by a pool of --threads encoder threads started once, into per-thread buffers kept across
//    requests; every engine context is created at start-up.
#include <arpa/inet.h>
#include <dirent.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <omp.h>
#include <poll.h>
#include <sys/socket.h>
#include <sys/stat.h>
#include <sys/un.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <csignal>
#include <deque>
#include <functional>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/gsj.h"
#include "../../../include/gsjd.h"
#include "../../../include/gsp_protocol.h"
#include "load.h"
#include "rows.h"

namespace gsjd {
namespace {

using Clock = std::chrono::steady_clock;
double secs_since(Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); }

struct Config {
  std::string socket = "/tmp/gpujoind.sock", tcp, token, data_dir = ".";
  int device = 0, workers = 2, threads = 16;
  int refine_mode = GSJ_REFINE_FILTERED;
  double mem_budget_gb = 0;   // scratch budget shared by running requests (0: half of the free memory at first use)
  uint32_t stream_batch = 0;   // probe geometries per engine batch when rows are streamed (0: one batch)
  int gpu_encode = 1;           // rows encoded on the device (gsj_encode_rows) when they are sent from the engine's thread
  std::string snapshot_dir;     // prepared layers saved here after LOAD and restored at start-up (empty: off)
  int tune = 0;                 // run the refinement autotuner on each LOADed polygon layer of >= kTuneGeoms geometries
};
Config g_cfg;
// the refinement launch shape every context takes when it is leased (set by the autotuner at LOAD, --tune)
std::mutex g_shape_m;
bool g_shape_set = false;
gsj_refine_shape g_shape{};
constexpr uint64_t kTuneGeoms = 100000;
std::atomic<bool> g_stop{false};

void logf(const char* fmt, ...) {
  char ts[32];
  const time_t now = time(nullptr);
  struct tm tmv;
  localtime_r(&now, &tmv);
  strftime(ts, sizeof ts, "%Y-%m-%d %H:%M:%S", &tmv);
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "[%s] ", ts);
  vfprintf(stderr, fmt, ap);
  fputc('\n', stderr);
  va_end(ap);
}

// ---- JSON text -------------------------------------------------------------------------------------------------
std::string jquote(const std::string& s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    if (c == '"' || c == '\\') { o += '\\'; o += (char)c; }
    else if (c < 0x20) { char b[8]; snprintf(b, sizeof b, "\\u%04x", c); o += b; }
    else o += (char)c;
  }
  return o + "\"";
}
std::string jnum(double x) {
  if (!std::isfinite(x)) return "null";
  char b[64];
  snprintf(b, sizeof b, "%.6g", x);
  return b;
}
class Json {
 public:
  Json& key(const char* k) { s_ += first_ ? "" : ","; first_ = false; s_ += jquote(k) + ":"; return *this; }
  Json& str(const char* k, const std::string& v) { return key(k).raw(jquote(v)); }
  Json& num(const char* k, double v) { return key(k).raw(jnum(v)); }
  Json& u64(const char* k, uint64_t v) { return key(k).raw(std::to_string(v)); }
  Json& boolean(const char* k, bool v) { return key(k).raw(v ? "true" : "false"); }
  Json& raw(const std::string& v) { s_ += v; return *this; }
  std::string done() const { return s_ + "}"; }

 private:
  std::string s_ = "{";
  bool first_ = true;
};

// ---- engine contexts and admission ------------------------------------------------------------------------------
// Two pools of contexts on one device, created on first use (the daemon starts without touching the GPU): small
// requests (probe layers of at most kSmallGeoms geometries) run on high-priority streams, so their kernels get SMs
// ahead of a large request's as its blocks retire; large requests run on normal-priority streams. In each pool a
// request is admitted in arrival order once a context is free and its scratch estimate fits in the pool's budget
// beside the running requests (a request larger than the whole budget runs alone).
constexpr uint64_t kSmallGeoms = 16384;
class GpuPool {
 public:
  GpuPool(int high, int share) : high_(high), share_(share) {}
  gsj_ctx* acquire(uint64_t est) {
    std::unique_lock<std::mutex> lk(m_);
    const uint64_t ticket = next_++;
    cv_.wait(lk, [&] {
      return ticket == serving_ && (!free_.empty() || created_ < size()) && (busy_ == 0 || budget_ == 0 || used_ + est <= budget_);
    });
    serving_++;
    gsj_ctx* c = nullptr;
    if (!free_.empty()) { c = free_.back(); free_.pop_back(); }
    else {
      const int rc = create(&c);
      if (rc) {
        cv_.notify_all();
        throw std::runtime_error("no usable CUDA device " + std::to_string(g_cfg.device) + " (gsj_ctx_create: " + std::to_string(rc) + ")");
      }
    }
    busy_++;
    used_ += est;
    cv_.notify_all();
    lk.unlock();
    {
      std::lock_guard<std::mutex> sl(g_shape_m);
      if (g_shape_set) gsj_set_refine_shape(c, &g_shape);
    }
    return c;
  }
  void release(gsj_ctx* c, uint64_t est) {
    std::lock_guard<std::mutex> lk(m_);
    free_.push_back(c);
    busy_--;
    used_ -= est;
    cv_.notify_all();
  }
  // Every context of the pool at start-up: creating one later happens under the pool lock, in front of the
  // request that needed it. Best effort: without a usable device the first request reports the error.
  void prewarm() {
    std::lock_guard<std::mutex> lk(m_);
    while (created_ < size()) {
      gsj_ctx* c = nullptr;
      const int rc = create(&c);
      if (rc) { logf("no engine context at start-up (gsj_ctx_create: %d); creating on first use", rc); return; }
      free_.push_back(c);
    }
  }
  void counts(int* busy, uint64_t* queued, uint64_t* used, uint64_t* budget) {
    std::lock_guard<std::mutex> lk(m_);
    *busy += busy_;
    *queued += next_ - serving_;
    *used += used_;
    *budget += budget_;
  }

 private:
  int size() const { return std::max(1, share_ == 0 ? g_cfg.workers / 2 : g_cfg.workers - g_cfg.workers / 2); }
  int create(gsj_ctx** c) {   // caller holds m_
    const int rc = gsj_ctx_create_prio(g_cfg.device, high_, c);
    if (rc) return rc;
    created_++;
    if (!budget_set_) {
      uint64_t fr = 0, tot = 0;
      gsj_ctx_mem_info(*c, &fr, &tot, nullptr);
      const uint64_t all = g_cfg.mem_budget_gb > 0 ? (uint64_t)(g_cfg.mem_budget_gb * 1073741824.0) : fr / 2;
      budget_ = all / 2;
      budget_set_ = true;
    }
    return 0;
  }
  int high_, share_;
  std::mutex m_;
  std::condition_variable cv_;
  std::vector<gsj_ctx*> free_;
  int created_ = 0, busy_ = 0;
  uint64_t next_ = 0, serving_ = 0, used_ = 0, budget_ = 0;
  bool budget_set_ = false;
};
GpuPool g_pool_small(1, 0), g_pool_large(0, 1);

class Lease {
 public:
  // small: the request's probe layer has at most kSmallGeoms geometries
  explicit Lease(uint64_t est = 0, bool small = false)
      : est_(est), pool_(small ? g_pool_small : g_pool_large), c_(pool_.acquire(est)) {}
  ~Lease() { pool_.release(c_, est_); }
  gsj_ctx* get() const { return c_; }
  Lease(const Lease&) = delete;
  Lease& operator=(const Lease&) = delete;

 private:
  uint64_t est_;
  GpuPool& pool_;
  gsj_ctx* c_;
};

void check(gsj_ctx* c, int rc, const char* what) {
  if (rc) throw std::runtime_error(std::string(what) + ": " + gsj_last_error(c));
}

// ---- layers -------------------------------------------------------------------------------------------------------
struct Layer {
  std::string name, kind, source;
  int subdiv = 0;
  bool deduped = false;
  IdTable ids;
  uint64_t rows = 0, skipped = 0, n_distinct = 0, gpu_geoms = 0, verts = 0, gpu_bytes = 0;
  std::vector<uint64_t> moff;
  std::vector<uint32_t> midx;
  gsj_layer* h = nullptr;
  gsj_rowset* rs = nullptr;   // row ids (and members) on the device, for encoding rows there
  double copy_s = 0, prep_s = 0, upload_s = 0;

  Members members() const { return deduped ? Members{moff.data(), midx.data()} : Members{}; }
  bool points() const { return kind == "point"; }
  ~Layer() {
    if (rs) gsj_rowset_free(rs);
    if (h) gsj_layer_free(nullptr, h);
  }
  std::string json() const {   // Layer::json, gpujoind.cu:81-86
    return Json().str("layer", name).str("kind", kind).str("source", source).u64("rows", rows).u64("skipped", skipped)
        .u64("distinct", n_distinct).u64("gpu_geoms", gpu_geoms).u64("vertices", verts).u64("subdivide", (uint64_t)subdiv)
        .boolean("dedup", deduped).num("gpu_mb", gpu_bytes / 1048576.0).num("copy_s", copy_s).num("prepare_s", prep_s)
        .num("upload_s", upload_s).done();
  }
};

// Scratch estimate of a join of probe layer P against build layer R: candidate pairs (one 8-byte pair, the
// refinement outputs and the compaction buffers, ~96 bytes each) at ~24 candidates per probe geometry, plus the
// per-call fixed buffers. Generous on purpose: it only orders admission.
uint64_t scratch_estimate(const Layer& P, const Layer& R) {
  (void)R;
  return (64ull << 20) + P.gpu_geoms * 24ull * 96ull;
}

std::mutex g_reg;
std::map<std::string, std::shared_ptr<Layer>> g_layers;

std::shared_ptr<Layer> get_layer(const std::string& n) {
  std::lock_guard<std::mutex> g(g_reg);
  auto it = g_layers.find(n);
  if (it == g_layers.end()) throw std::runtime_error("no such layer: " + n);
  return it->second;
}

// LOAD's table argument: a file inside the data directory.
std::string resolve_path(const std::string& p) {
  if (p.empty()) throw std::runtime_error("LOAD needs a file path as its table argument");
  const std::string full = p[0] == '/' ? p : g_cfg.data_dir + "/" + p;
  char rp[PATH_MAX], rd[PATH_MAX];
  if (!realpath(full.c_str(), rp)) throw std::runtime_error("cannot open " + p + ": " + strerror(errno));
  if (!realpath(g_cfg.data_dir.c_str(), rd)) throw std::runtime_error("bad --data-dir");
  const std::string a = rp, d = rd;
  if (a.compare(0, d.size(), d) != 0 || (a.size() > d.size() && a[d.size()] != '/' && d != "/"))
    throw std::runtime_error("LOAD reads files inside the data directory only: " + p);
  return a;
}

template <class T> struct HostArray {   // library-allocated host arrays (gsj_dedup / gsj_subdivide outputs)
  T* p = nullptr;
  ~HostArray() { if (p) gsj_host_free(p); }
};

// ---- prepared-layer snapshots: a restart restores every loaded layer without reading, deduplicating or
// subdividing its source again. One file per layer: header, ids, members, then the arrays as uploaded. ----
constexpr char kSnapMagic[8] = {'G', 'S', 'J', 'S', 'N', 'A', 'P', '1'};
struct SnapArrays {   // what gsj_layer_upload_* received
  uint64_t n = 0, nr = 0, nv = 0;
  const uint64_t* gro = nullptr; const uint64_t* rvo = nullptr; const double* xy = nullptr;
  const uint32_t* parent = nullptr; const uint8_t* syn = nullptr;
};
std::string snapshot_path(const std::string& name) {
  static const char* hx = "0123456789abcdef";
  std::string f;
  for (unsigned char ch : name) { f += hx[ch >> 4]; f += hx[ch & 15]; }
  return g_cfg.snapshot_dir + "/" + f + ".gsnap";
}
void write_snapshot(const Layer& L, const SnapArrays& A) {
  const std::string path = snapshot_path(L.name), tmp = path + ".tmp";
  FILE* f = fopen(tmp.c_str(), "wb");
  if (!f) { logf("snapshot %s: cannot write %s", L.name.c_str(), tmp.c_str()); return; }
  bool ok = true;
  auto put = [&](const void* p, size_t n) { if (ok && n && fwrite(p, 1, n, f) != n) ok = false; };
  auto put64 = [&](uint64_t v) { put(&v, 8); };
  auto putstr = [&](const std::string& v) { put64(v.size()); put(v.data(), v.size()); };
  put(kSnapMagic, 8);
  put64(L.points() ? 1 : 0); put64((uint64_t)L.subdiv); put64(L.deduped ? 1 : 0);
  put64(L.rows); put64(L.skipped); put64(L.n_distinct); put64(A.n); put64(A.nr); put64(A.nv);
  putstr(L.name); putstr(L.source);
  put64(L.ids.buf.size()); put(L.ids.buf.data(), L.ids.buf.size()); put(L.ids.off.data(), L.ids.off.size() * 8);
  if (L.deduped) { put(L.moff.data(), L.moff.size() * 8); put(L.midx.data(), L.midx.size() * 4); }
  if (L.points()) {
    put(A.xy, A.n * 16);
  } else {
    put(A.gro, (A.n + 1) * 8); put(A.rvo, (A.nr + 1) * 8); put(A.xy, A.nv * 16);
    put64(A.parent ? 1 : 0);
    if (A.parent) { put(A.parent, A.n * 4); put(A.syn, A.nv); }
  }
  ok = fclose(f) == 0 && ok;
  if (!ok || rename(tmp.c_str(), path.c_str()) != 0) { remove(tmp.c_str()); logf("snapshot %s: write failed", L.name.c_str()); }
}
void register_layer(const std::shared_ptr<Layer>& L) {
  std::shared_ptr<Layer> old;
  std::lock_guard<std::mutex> g(g_reg);
  auto& slot = g_layers[L->name];
  old = slot;
  slot = L;
}
// restores one snapshot; returns "" or the reason it was skipped
std::string restore_snapshot(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return "cannot open";
  std::unique_ptr<FILE, int (*)(FILE*)> guard(f, fclose);
  bool ok = true;
  auto get = [&](void* p, size_t n) { if (ok && n && fread(p, 1, n, f) != n) ok = false; };
  auto get64 = [&]() { uint64_t v = 0; get(&v, 8); return v; };
  auto getstr = [&]() { std::string v(std::min<uint64_t>(get64(), 1 << 20), '\0'); get(&v[0], v.size()); return v; };
  char mg[8] = {0};
  get(mg, 8);
  if (!ok || std::memcmp(mg, kSnapMagic, 8) != 0) return "not a snapshot";
  auto L = std::make_shared<Layer>();
  const bool pts = get64() != 0;
  L->subdiv = (int)get64(); L->deduped = get64() != 0;
  L->rows = get64(); L->skipped = get64(); L->n_distinct = get64();
  const uint64_t n = get64(), nr = get64(), nv = get64();
  L->name = getstr(); L->source = getstr() + " (snapshot)";
  if (!ok || L->rows == 0 || L->rows > (1ull << 32) || n > (1ull << 32) || nv > (1ull << 40)) return "bad header";
  const uint64_t blob = get64();
  if (!ok || blob > (1ull << 36)) return "bad id table";
  L->ids.buf.resize(blob); get(&L->ids.buf[0], blob);
  L->ids.off.resize(L->rows + 1); get(L->ids.off.data(), (L->rows + 1) * 8);
  if (!ok || L->ids.off[0] != 0 || L->ids.off[L->rows] != blob) return "bad id table";
  if (L->deduped) {
    L->moff.resize(L->n_distinct + 1); get(L->moff.data(), L->moff.size() * 8);
    L->midx.resize(L->rows); get(L->midx.data(), L->midx.size() * 4);
  }
  // the big arrays are read into uninitialised buffers (a zero-filled vector would write them twice)
  std::unique_ptr<uint64_t[]> gro, rvo;
  std::unique_ptr<double[]> xy;
  std::unique_ptr<uint32_t[]> parent;
  std::unique_ptr<uint8_t[]> syn;
  Lease lease;
  if (pts) {
    L->kind = "point"; L->gpu_geoms = L->verts = n;
    xy.reset(new double[2 * n]); get(xy.get(), n * 16);
    if (!ok) return "truncated";
    check(lease.get(), gsj_layer_upload_points(lease.get(), n, xy.get(), &L->h), "upload");
  } else {
    L->kind = "polygon"; L->gpu_geoms = n; L->verts = nv;
    gro.reset(new uint64_t[n + 1]); rvo.reset(new uint64_t[nr + 1]); xy.reset(new double[2 * nv]);
    get(gro.get(), (n + 1) * 8); get(rvo.get(), (nr + 1) * 8); get(xy.get(), nv * 16);
    if (get64()) { parent.reset(new uint32_t[n]); syn.reset(new uint8_t[nv]); get(parent.get(), n * 4); get(syn.get(), nv); }
    if (!ok) return "truncated";
    if (gro[0] != 0 || gro[n] != nr || rvo[0] != 0 || rvo[nr] != nv) return "inconsistent offsets";
    check(lease.get(), gsj_layer_upload_polygons(lease.get(), n, nr, nv, gro.get(), rvo.get(), xy.get(), parent.get(), syn.get(), &L->h), "upload");
  }
  check(lease.get(), gsj_rowset_upload(lease.get(), L->n_distinct, L->deduped ? L->moff.data() : nullptr, L->deduped ? L->midx.data() : nullptr,
                                       L->rows, L->ids.buf.data(), L->ids.off.data(), &L->rs), "row ids upload");
  gsj_layer_info info;
  gsj_layer_get_info(L->h, &info);
  L->gpu_bytes = info.device_bytes;
  register_layer(L);
  logf("restored %s from %s: %s", L->name.c_str(), path.c_str(), L->json().c_str());
  return "";
}
void restore_snapshots() {
  if (g_cfg.snapshot_dir.empty()) return;
  DIR* d = opendir(g_cfg.snapshot_dir.c_str());
  if (!d) { logf("snapshot dir %s: cannot open", g_cfg.snapshot_dir.c_str()); return; }
  std::vector<std::string> files;
  while (dirent* e = readdir(d)) {
    const std::string nm = e->d_name;
    if (nm.size() > 6 && nm.compare(nm.size() - 6, 6, ".gsnap") == 0) files.push_back(g_cfg.snapshot_dir + "/" + nm);
  }
  closedir(d);
  std::sort(files.begin(), files.end());
  for (const auto& fpath : files) {
    try {
      const std::string why = restore_snapshot(fpath);
      if (!why.empty()) logf("snapshot %s skipped: %s", fpath.c_str(), why.c_str());
    } catch (const std::exception& ex) {
      logf("snapshot %s skipped: %s", fpath.c_str(), ex.what());
    }
  }
}

std::string build_layer(const std::string& name, const std::string& path, int subdiv, bool dedup) {
  auto t0 = Clock::now();
  LoadedLayer ld;
  const std::string err = load_layer_file(path, ld);
  if (!err.empty()) throw std::runtime_error("load failed: " + err);
  auto L = std::make_shared<Layer>();
  L->name = name; L->subdiv = subdiv; L->source = "file " + path; L->copy_s = secs_since(t0);
  L->rows = ld.ids.size();
  L->skipped = ld.skipped_null + ld.skipped_type + ld.skipped_empty;
  L->ids = std::move(ld.ids);
  logf("load %s: %llu rows in %.2fs (skipped null=%llu type=%llu empty=%llu)", name.c_str(), (unsigned long long)L->rows, L->copy_s,
       (unsigned long long)ld.skipped_null, (unsigned long long)ld.skipped_type, (unsigned long long)ld.skipped_empty);
  t0 = Clock::now();
  if (ld.is_points) {
    L->kind = "point"; L->n_distinct = L->gpu_geoms = L->verts = L->rows;
    if (L->rows == 0) throw std::runtime_error("layer has no rows");
    Lease lease;
    auto t1 = Clock::now();
    check(lease.get(), gsj_layer_upload_points(lease.get(), L->rows, ld.xy.data(), &L->h), "upload");
    L->upload_s = secs_since(t1);
    if (!g_cfg.snapshot_dir.empty()) {
      SnapArrays A; A.n = L->rows; A.xy = ld.xy.data();
      write_snapshot(*L, A);
    }
  } else {
    L->kind = "polygon";
    const uint64_t n = ld.gro.size() - 1;
    if (n == 0) throw std::runtime_error("layer has no polygonal rows");
    uint64_t bn = n, bnr = ld.rvo.size() - 1, bnv = ld.xy.size() / 2;
    const uint64_t* gro = ld.gro.data();
    const uint64_t* rvo = ld.rvo.data();
    const double* xy = ld.xy.data();
    HostArray<uint64_t> dgro, drvo, dmoff, sgro, srvo;
    HostArray<double> dxy, sxy;
    HostArray<uint32_t> dmidx, spar;
    HostArray<uint8_t> ssyn;
    Lease lease;
    if (dedup) {   // identical geometries once, rows expand to members (dedup_set, first-occurrence order; on the GPU)
      uint64_t un, unr, unv;
      check(lease.get(), gsj_dedup_gpu(lease.get(), bn, bnr, bnv, gro, rvo, xy, 0, &un, &unr, &unv, &dgro.p, &drvo.p, &dxy.p, &dmoff.p, &dmidx.p),
            "dedup");
      L->deduped = true;
      L->moff.assign(dmoff.p, dmoff.p + un + 1);
      L->midx.assign(dmidx.p, dmidx.p + n);
      bn = un; bnr = unr; bnv = unv; gro = dgro.p; rvo = drvo.p; xy = dxy.p;
    }
    L->n_distinct = bn;
    if (subdiv > 0) {   // on the GPU (subdivide_set's pieces, bit for bit)
      uint64_t pn, pnr, pnv;
      check(lease.get(), gsj_subdivide_gpu(lease.get(), bn, bnr, bnv, gro, rvo, xy, subdiv, &pn, &pnr, &pnv, &sgro.p, &srvo.p, &sxy.p, &spar.p, &ssyn.p),
            "subdivide");
      bn = pn; bnr = pnr; bnv = pnv; gro = sgro.p; rvo = srvo.p; xy = sxy.p;
    }
    L->gpu_geoms = bn; L->verts = bnv;
    L->prep_s = secs_since(t0);
    uint64_t fr = 0, tot = 0;
    check(lease.get(), gsj_ctx_mem_info(lease.get(), &fr, &tot, nullptr), "memory query");
    const uint64_t need = bnv * 16 + bnr * 8 + bn * 120 + bnv / 8;   // vertices, rings, per-geometry arrays + LBVH
    if (need + (2ull << 30) > fr)
      throw std::runtime_error("not enough GPU memory: need ~" + std::to_string(need >> 20) + " MB, free " + std::to_string(fr >> 20) + " MB");
    auto t1 = Clock::now();
    check(lease.get(), gsj_layer_upload_polygons(lease.get(), bn, bnr, bnv, gro, rvo, xy, subdiv > 0 ? spar.p : nullptr,
                                                 subdiv > 0 ? ssyn.p : nullptr, &L->h), "upload");
    L->upload_s = secs_since(t1);
    if (g_cfg.tune && bn >= kTuneGeoms) {   // launch shape for joins against this layer, from a sample of its self-join
      gsj_refine_params rp;
      gsj_refine_params_default(&rp);
      gsj_tune_result tr;
      // run and runs stay: their product bounds how long a refinement block holds an SM while other requests'
      // kernels (high-priority streams) wait for one
      const int rc = gsj_tune_refine(lease.get(), L->h, L->h, &rp, g_cfg.refine_mode, 1, 1u << 20, GSJ_TUNE_KEEP_RUN | GSJ_TUNE_KEEP_RUNS, &tr);
      if (rc) logf("tune %s: %s", name.c_str(), gsj_last_error(lease.get()));
      else {
        std::lock_guard<std::mutex> sl(g_shape_m);
        g_shape = tr.best;
        g_shape_set = true;
        logf("tune %s: shape run=%d runs=%d bin_edges=%d scratch_warps_per_sm=%d, %.2f -> %.2f ms on %llu pairs (%u shapes)", name.c_str(),
             tr.best.run, tr.best.runs, tr.best.bin_edges, tr.best.scratch_warps_per_sm, tr.start_ms, tr.best_ms, (unsigned long long)tr.sample_pairs,
             tr.shapes_tried);
      }
    }
    if (!g_cfg.snapshot_dir.empty()) {   // the arrays as uploaded (after dedup / subdivision), with the ids and members
      SnapArrays A; A.n = bn; A.nr = bnr; A.nv = bnv; A.gro = gro; A.rvo = rvo; A.xy = xy;
      if (subdiv > 0) { A.parent = spar.p; A.syn = ssyn.p; }
      write_snapshot(*L, A);
    }
  }
  {
    Lease lease;
    check(lease.get(), gsj_rowset_upload(lease.get(), L->n_distinct, L->deduped ? L->moff.data() : nullptr, L->deduped ? L->midx.data() : nullptr,
                                         L->rows, L->ids.buf.data(), L->ids.off.data(), &L->rs), "row ids upload");
  }
  gsj_layer_info info;
  gsj_layer_get_info(L->h, &info);
  L->gpu_bytes = info.device_bytes;
  const std::string js = L->json();
  logf("load %s: ready %s", name.c_str(), js.c_str());
  register_layer(L);
  return js;
}

// ---- connection ---------------------------------------------------------------------------------------------------
struct Conn {
  int fd;
  volatile int broken = 0;   // the client went away: the engine stops between batches (JoinOpts::cancel)
  bool streaming = false;    // a result stream started: errors go out as GSP_FRAME_ERR
  bool read_full(void* p, size_t n) {
    char* c = static_cast<char*>(p);
    while (n) {
      const ssize_t r = ::read(fd, c, n);
      if (r <= 0) { if (r < 0 && errno == EINTR) continue; return false; }
      c += r; n -= (size_t)r;
    }
    return true;
  }
  bool write_full(const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    while (n && !broken) {
      const ssize_t r = ::send(fd, c, n, MSG_NOSIGNAL);
      if (r <= 0) { if (r < 0 && errno == EINTR) continue; broken = 1; return false; }
      c += r; n -= (size_t)r;
    }
    return !broken;
  }
  bool u32(uint32_t v) { return write_full(&v, 4); }
  bool str(const std::string& s) { return u32((uint32_t)s.size()) && write_full(s.data(), s.size()); }
  void ok_json(const std::string& j) { u32(GSP_OK); str(j); }
  void error(const std::string& m) { u32(GSP_ERR); str(m); }
  void end_stream(const std::string& stats) { u32(0); str(stats); }
};

// Encoder threads shared by all requests (started once: connection threads are short-lived, so a per-call thread
// team would be created afresh for every request). run(nch, f) calls f(0 .. nch-1) on the pool and the calling
// thread and returns when all are done.
class EncodePool {
 public:
  void start(int n) {
    for (int i = 0; i < n; i++) std::thread([this] { loop(); }).detach();
    threads_ = n;
  }
  template <class F> void run(uint64_t nch, F&& f) {
    if (threads_ == 0 || nch < 2) { for (uint64_t k = 0; k < nch; k++) f(k); return; }
    Job j;
    j.fn = [&f](uint64_t k) { f(k); };
    j.n = nch;
    { std::lock_guard<std::mutex> l(m_); q_.push_back(&j); }
    cv_.notify_all();
    work(j);
    std::unique_lock<std::mutex> l(m_);
    done_cv_.wait(l, [&] { return j.finished == j.n && j.helpers == 0; });
    drop(&j);   // under the same lock as the check: no helper can pick the job up any more
  }

 private:
  struct Job { std::function<void(uint64_t)> fn; uint64_t n = 0, finished = 0; std::atomic<uint64_t> next{0}; int helpers = 0; };
  void drop(Job* j) {   // caller holds m_
    for (auto it = q_.begin(); it != q_.end(); ++it)
      if (*it == j) { q_.erase(it); return; }
  }
  void work(Job& j) {
    for (;;) {
      const uint64_t k = j.next.fetch_add(1);
      if (k >= j.n) return;
      j.fn(k);
      std::lock_guard<std::mutex> l(m_);
      if (++j.finished == j.n) done_cv_.notify_all();
    }
  }
  void loop() {
    for (;;) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return !q_.empty(); });
        j = q_.front();
        j->helpers++;
      }
      work(*j);
      std::lock_guard<std::mutex> l(m_);
      drop(j);   // its chunks are all taken
      j->helpers--;
      done_cv_.notify_all();
    }
  }
  int threads_ = 0;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  std::deque<Job*> q_;
};
EncodePool& g_encode = *new EncodePool;   // never destroyed: its detached threads wait on it until exit

// Encode rows of n items into independent runs of complete frames and send them in order (send_parallel,
// gpujoind.cu:192-206): in parallel on the encoder threads for a whole join's rows, on the calling thread for one
// streamed batch (the GPU runs the next batch meanwhile). enc(i, FrameWriter&) writes the rows of item i.
// enc_s / wr_s (optional) accumulate the encoding and writing seconds.
thread_local bool t_sequential_encode = false;
template <class Enc> uint64_t send_rows(Conn& c, uint64_t n, Enc&& enc, double* enc_s = nullptr, double* wr_s = nullptr) {
  if (!n || c.broken) return 0;
  const auto t0 = Clock::now();
  const bool par = !t_sequential_encode && n >= 4096;
  const uint64_t nch = par ? std::min<uint64_t>(n, (uint64_t)std::max(1, g_cfg.threads) * 4) : 1;
  thread_local std::vector<FrameWriter> t_fw;   // kept with their capacity: steady-state requests touch no new pages
  if (t_fw.size() < nch) t_fw.resize(nch);
  FrameWriter* fw = t_fw.data();
  auto one = [&](uint64_t k) {
    const uint64_t i0 = n * k / nch, i1 = n * (k + 1) / nch;
    fw[k].reset();
    fw[k].reserve((i1 - i0) * 48);
    fw[k].begin();
    for (uint64_t i = i0; i < i1; i++) enc(i, fw[k]);
    fw[k].finish();
  };
  if (par) g_encode.run(nch, one);
  else one(0);
  const auto t1 = Clock::now();
  uint64_t rows = 0;
  for (uint64_t k = 0; k < nch; k++) {
    if (!c.write_full(fw[k].data(), fw[k].size())) break;
    rows += fw[k].rows;
  }
  if (enc_s) *enc_s += std::chrono::duration<double>(t1 - t0).count();
  if (wr_s) *wr_s += secs_since(t1);
  return rows;
}

// Rows of finished engine batches, sent either at once (sync: the consumer reads the engine's host buffers in
// the sink) or by a sender thread (the sink copies the batch out, since the engine reuses its buffers, and
// returns so that the GPU starts the next batch while this one is encoded and written). At most kMaxQueued
// batches wait; a sink that would exceed that blocks until the sender catches up.
class Streamer {
 public:
  using Fn = std::function<void(const uint32_t* p, const double* ar, const uint32_t* code, const uint8_t* wh, uint64_t n)>;
  Streamer(bool pipelined, Fn fn) : fn_(std::move(fn)), on_(pipelined) {
    if (on_) th_ = std::thread([this] { t_sequential_encode = true; run(); });
  }
  ~Streamer() { finish(); }
  Streamer(const Streamer&) = delete;
  Streamer& operator=(const Streamer&) = delete;

  void push(const uint32_t* p, const double* ar, const uint32_t* code, const uint8_t* wh, uint64_t n) {
    if (!on_) { fn_(p, ar, code, wh, n); return; }
    Batch b;
    b.n = n;
    b.p.assign(p, p + 2 * n);
    if (ar) b.ar.assign(ar, ar + n);
    if (code) b.code.assign(code, code + n);
    if (wh) b.wh.assign(wh, wh + n);
    std::unique_lock<std::mutex> l(m_);
    room_.wait(l, [&] { return q_.size() < kMaxQueued; });
    q_.push_back(std::move(b));
    ready_.notify_one();
  }
  void finish() {   // every pushed batch sent (or dropped by the consumer on a broken connection)
    if (!on_ || !th_.joinable()) return;
    { std::lock_guard<std::mutex> l(m_); done_ = true; }
    ready_.notify_one();
    th_.join();
  }

 private:
  struct Batch { std::vector<uint32_t> p; std::vector<double> ar; std::vector<uint32_t> code; std::vector<uint8_t> wh; uint64_t n = 0; };
  static constexpr size_t kMaxQueued = 4;
  void run() {
    for (;;) {
      Batch b;
      {
        std::unique_lock<std::mutex> l(m_);
        ready_.wait(l, [&] { return done_ || !q_.empty(); });
        if (q_.empty()) return;
        b = std::move(q_.front());
        q_.pop_front();
        room_.notify_one();
      }
      fn_(b.p.data(), b.ar.empty() ? nullptr : b.ar.data(), b.code.empty() ? nullptr : b.code.data(), b.wh.empty() ? nullptr : b.wh.data(), b.n);
    }
  }
  Fn fn_;
  bool on_;
  std::thread th_;
  std::mutex m_;
  std::condition_variable ready_, room_;
  std::deque<Batch> q_;
  bool done_ = false;
};

// send_rows with the request's encode / write seconds accumulated in its run record
template <class Run, class Enc> uint64_t send_rows_acc(Run& r, Conn& c, uint64_t n, Enc&& enc) {
  return send_rows(c, n, std::forward<Enc>(enc), &r.enc_s, &r.wr_s);
}

constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

// Rows encoded on the device (gsj_encode_rows: the same rows, whole frames) on the request's context, written as
// they come back. Used when the engine's sink runs on the request's thread (not with streamed batches, whose
// sender thread cannot share the context).
struct GpuWrite { Conn* c; double* wr_s; };
int gpu_frames_sink(void* u, const uint8_t* bytes, uint64_t nb, uint64_t) {
  auto* g = static_cast<GpuWrite*>(u);
  const auto t = Clock::now();
  const bool ok = g->c->write_full(bytes, nb);
  *g->wr_s += secs_since(t);
  return ok ? 0 : 1;
}
uint64_t gpu_rows(gsj_ctx* ctx, Conn& c, const Layer& P, const Layer& Q, int mode, bool same, bool distinct, bool swapped, double value,
                  const std::string& pattern, const uint32_t* p, const double* ar, const uint32_t* code, const uint8_t* wh, uint64_t n,
                  double* enc_s, double* wr_s) {
  if (!n || c.broken) return 0;
  gsj_encode_spec sp;
  sp.mode = mode; sp.same = same; sp.distinct = distinct; sp.swapped = swapped; sp.point_value = value;
  std::memset(sp.pattern, 0, sizeof sp.pattern);
  std::memcpy(sp.pattern, pattern.data(), std::min<size_t>(pattern.size(), 9));
  GpuWrite g{&c, wr_s};
  const double w0 = *wr_s;
  const auto t0 = Clock::now();
  uint64_t rows = 0;
  const int rc = gsj_encode_rows(ctx, P.rs, Q.rs, &sp, p, ar, code, wh, n, gpu_frames_sink, &g, &rows);
  *enc_s += secs_since(t0) - (*wr_s - w0);
  if (rc && rc != GSJ_ERR_SINK) throw std::runtime_error(std::string("row encoding: ") + gsj_last_error(ctx));
  return rows;
}
// relate(point, polygon) for a point inside / on the boundary (DE9IM_PT_INTERIOR / _BOUNDARY, engine.cuh:337-338)
constexpr uint32_t kPtInterior = 1u | (3u << 12) | (2u << 14) | (3u << 16);   // 0FFFFF212
constexpr uint32_t kPtBoundary = (1u << 2) | (3u << 12) | (2u << 14) | (3u << 16);   // F0FFFF212

bool self_pairs_arg(const std::string& s) {
  if (s != "all" && s != "distinct") throw std::runtime_error("self_pairs must be 'all' or 'distinct'");
  return s == "distinct";
}

// The engine call failed: the client going away ends the request quietly, anything else is an error.
void engine_status(Conn& c, gsj_ctx* ctx, int rc, const char* what) {
  if (!rc) return;
  if (c.broken && (rc == GSJ_ERR_SINK || rc == GSJ_ERR_CANCELLED)) return;
  throw std::runtime_error(std::string(what) + ": " + gsj_last_error(ctx));
}

std::string with_stats_only(const std::string& stats, bool want_area, double area_sum) {
  return stats.substr(0, stats.size() - 1) + ",\"stats_only\":true" + (want_area ? ",\"area_sum\":" + jnum(area_sum) : std::string()) + "}";
}

// ---- JOIN (op_join, gpujoind.cu:210-290) ----------------------------------------------------------------------------
struct JoinRun {
  Conn* c;
  const Layer *A, *B;   // engine order: A probe (points when one side is points), B build
  const Layer *LA, *LB; // output order
  bool same, distinct, want_area, stats_only, swapped;
  uint64_t total = 0;
  double area_sum = 0, host_s = 0, enc_s = 0, wr_s = 0;
  Streamer* out = nullptr;
  gsj_ctx* gctx = nullptr;   // set: rows encoded on the device
};

void join_rows(JoinRun& J, const uint32_t* p, const double* ar, uint64_t n) {
  const auto th = Clock::now();
  const Members MA = J.A->members(), MB = J.B->members();
  if (J.stats_only) {
    uint64_t t = 0;
    double as = 0;
#pragma omp parallel for num_threads(g_cfg.threads) reduction(+ : t, as)
    for (int64_t i = 0; i < (int64_t)n; i++) {
      const uint64_t k = pair_row_count(p[2 * i], p[2 * i + 1], MA, MB, J.same, J.distinct);
      t += k;
      if (ar) as += ar[i] * (double)k;
    }
    J.total += t; J.area_sum += as; J.host_s += secs_since(th);
    return;
  }
  const Layer& A = *J.A;
  const Layer& B = *J.B;
  if (J.gctx) {
    J.total += gpu_rows(J.gctx, *J.c, A, J.same ? A : B, GSJ_ENC_PAIRS, J.same, J.distinct, false, 0.0, "", p, ar, nullptr, nullptr, n,
                        &J.enc_s, &J.wr_s);
    J.host_s += secs_since(th);
    return;
  }
  J.total += send_rows_acc(J, *J.c, n, [&](uint64_t i, FrameWriter& f) {
    const double area = ar ? ar[i] : kNaN;
    pair_rows(p[2 * i], p[2 * i + 1], MA, MB, J.same, J.distinct, [&](uint32_t ra, uint32_t rb, bool) {
      const Layer& OB = J.same ? A : B;
      f.id(A.ids.data(ra), A.ids.len(ra)); f.id(OB.ids.data(rb), OB.ids.len(rb)); f.f64(area); f.row_done();
    });
  });
  J.host_s += secs_since(th);
}
int join_sink(void* u, const uint32_t* p, const double* ar, const uint32_t*, uint64_t n) {
  JoinRun& J = *static_cast<JoinRun*>(u);
  J.out->push(p, ar, nullptr, nullptr, n);
  return J.c->broken ? 1 : 0;
}

void join_points_rows(JoinRun& J, const uint32_t* p, uint64_t n) {
  const auto th = Clock::now();
  const Members MB = J.B->members();
  if (J.stats_only) {
    for (uint64_t i = 0; i < n; i++) J.total += MB.count(p[2 * i + 1]);
    J.host_s += secs_since(th);
    return;
  }
  if (J.gctx) {   // engine order: A points, B polygons
    J.total += gpu_rows(J.gctx, *J.c, *J.A, *J.B, GSJ_ENC_POINTS, false, false, J.swapped, J.want_area ? 0.0 : kNaN, "", p, nullptr, nullptr,
                        nullptr, n, &J.enc_s, &J.wr_s);
    J.host_s += secs_since(th);
    return;
  }
  J.total += send_rows_acc(J, *J.c, n, [&](uint64_t i, FrameWriter& f) {
    MB.each(p[2 * i + 1], [&](uint32_t rb) {
      uint32_t ra = p[2 * i];
      if (J.swapped) std::swap(ra, rb);
      f.id(J.LA->ids.data(ra), J.LA->ids.len(ra)); f.id(J.LB->ids.data(rb), J.LB->ids.len(rb));
      f.f64(J.want_area ? 0.0 : kNaN); f.row_done();
    });
  });
  J.host_s += secs_since(th);
}
int join_points_sink(void* u, const uint32_t* p, const uint8_t*, uint64_t n) {
  JoinRun& J = *static_cast<JoinRun*>(u);
  J.out->push(p, nullptr, nullptr, nullptr, n);
  return J.c->broken ? 1 : 0;
}

void op_join(Conn& c, const std::vector<std::string>& a) {
  if (a.size() < 4) throw std::runtime_error("JOIN needs layer_a, layer_b, want_area, self_pairs[, mode]");
  const bool stats_only = a.size() > 4 && a[4] == "stats";
  auto A = get_layer(a[0]), B = get_layer(a[1]);
  const bool want_area = a[2] == "1" || a[2] == "t" || a[2] == "true";
  const bool distinct = self_pairs_arg(a[3]);
  const bool same = A.get() == B.get();
  if (A->points() && B->points()) throw std::runtime_error("point x point joins are not supported");
  bool swapped = false;
  if (!A->points() && B->points()) { std::swap(A, B); swapped = true; }   // run as point x polygon
  Lease lease(scratch_estimate(*A, *B), A->gpu_geoms <= kSmallGeoms);
  gsj_ctx* ctx = lease.get();
  c.u32(GSP_OK);
  c.streaming = true;
  gsj_join_opts o;
  gsj_join_opts_default(&o);
  o.cancel = &c.broken;
  o.refine_mode = g_cfg.refine_mode;
  const auto t0 = Clock::now();
  JoinRun J{&c, A.get(), B.get(), swapped ? B.get() : A.get(), swapped ? A.get() : B.get(), same, distinct, want_area, stats_only, swapped};
  const bool pipe = !stats_only && g_cfg.stream_batch > 0;
  if (pipe) o.batch_q = g_cfg.stream_batch;
  Streamer out(pipe, [&](const uint32_t* p, const double* ar, const uint32_t*, const uint8_t*, uint64_t n) {
    if (J.A->points()) join_points_rows(J, p, n); else join_rows(J, p, ar, n);
  });
  J.out = &out;
  if (!pipe && g_cfg.gpu_encode && A->rs && B->rs) J.gctx = ctx;
  gsj_join_stats st{};
  std::string stats;
  if (A->points()) {
    const int rc = gsj_join_points(ctx, A->h, B->h, &o, join_points_sink, &J, &st);
    out.finish();
    engine_status(c, ctx, rc, "join");
    stats = Json().str("kind", "point_in_polygon").u64("candidates", st.candidates).u64("gpu_hits", st.hits).u64("rows", J.total)
        .num("traverse_ms", st.traverse_ms).num("refine_ms", st.refine_ms).num("host_encode_send_s", J.host_s).num("host_encode_s", J.enc_s).num("host_write_s", J.wr_s).num("total_s", secs_since(t0)).done();
  } else {
    gsj_refine_params rp;
    gsj_refine_params_default(&rp);
    rp.want_area = want_area ? 1 : 0;
    o.upper = same;   // self-join: each unordered pair once, mirrored by the row rules
    const int rc = gsj_join(ctx, A->h, B->h, &rp, &o, join_sink, &J, &st);
    out.finish();
    engine_status(c, ctx, rc, "join");
    stats = Json().str("kind", "polygon_polygon").u64("candidates", st.candidates).u64("gpu_hits", st.hits).u64("rows", J.total)
        .u64("heavy", st.heavy).num("traverse_ms", st.traverse_ms).num("refine_ms", st.refine_ms).num("compact_ms", st.compact_ms)
        .num("d2h_ms", st.copy_ms).num("host_encode_send_s", J.host_s).num("host_encode_s", J.enc_s).num("host_write_s", J.wr_s).num("total_s", secs_since(t0)).done();
  }
  if (stats_only) stats = with_stats_only(stats, want_area, J.area_sum);
  if (!c.broken) c.end_stream(stats);
  logf("join %s x %s area=%d: %s%s", a[0].c_str(), a[1].c_str(), (int)want_area, stats.c_str(), c.broken ? " (client went away)" : "");
}

// ---- CLUSTER (op_cluster, gpujoind.cu:293-320) ---------------------------------------------------------------------
void op_cluster(Conn& c, const std::vector<std::string>& a) {
  if (a.empty()) throw std::runtime_error("CLUSTER needs layer");
  auto L = get_layer(a[0]);
  if (L->points()) throw std::runtime_error("cluster needs a polygon layer");
  Lease lease(scratch_estimate(*L, *L));
  gsj_ctx* ctx = lease.get();
  const auto t0 = Clock::now();
  gsj_join_opts o;
  gsj_join_opts_default(&o);
  o.cancel = &c.broken;
  o.refine_mode = g_cfg.refine_mode;
  std::vector<uint32_t> root(L->n_distinct);
  gsj_join_stats st{};
  check(ctx, gsj_cluster(ctx, L->h, (uint32_t)L->n_distinct, &o, root.data(), &st), "cluster");
  const double uf_s = secs_since(t0);
  std::vector<uint32_t> label(L->rows);
  const uint32_t k = gsjd_cluster_labels((uint32_t)L->n_distinct, root.data(), L->rows, L->deduped ? L->moff.data() : nullptr,
                                         L->deduped ? L->midx.data() : nullptr, label.data());
  c.u32(GSP_OK);
  c.streaming = true;
  const uint64_t total = send_rows(c, L->rows, [&](uint64_t r, FrameWriter& f) {
    f.id(L->ids.data(r), L->ids.len(r)); f.u32(label[r]); f.row_done();
  });
  const std::string stats = Json().str("kind", "cluster_intersecting").u64("rows", total).u64("clusters", k).u64("candidates", st.candidates)
      .u64("edges", st.hits).num("traverse_ms", st.traverse_ms).num("refine_ms", st.refine_ms)
      .num("union_find_ms", std::max(0.0, uf_s * 1e3 - st.traverse_ms - st.refine_ms - st.compact_ms)).num("total_s", secs_since(t0)).done();
  if (!c.broken) c.end_stream(stats);
  logf("cluster %s: %s", a[0].c_str(), stats.c_str());
}

// ---- RELATE (op_relate, gpujoind.cu:323-388) ------------------------------------------------------------------------
struct RelateRun {
  Conn* c;
  const Layer *A, *B;
  bool same, distinct, swapped;
  std::string pat;
  uint64_t total = 0;
  double host_s = 0, enc_s = 0, wr_s = 0;
  Streamer* out = nullptr;
  gsj_ctx* gctx = nullptr;   // set: rows encoded on the device
};

void put_relate(FrameWriter& f, const RelateRun& R, const Layer& LA, uint32_t ra, const Layer& LB, uint32_t rb, uint32_t code) {
  if (!R.pat.empty() && !gsj_de9im_match(code, R.pat.c_str())) return;
  char m[9];
  gsj_de9im_str(code, m);
  f.id(LA.ids.data(ra), LA.ids.len(ra)); f.id(LB.ids.data(rb), LB.ids.len(rb)); f.raw(m, 9); f.row_done();
}

void relate_rows(RelateRun& R, const uint32_t* p, const uint32_t* code, uint64_t n) {
  const auto th = Clock::now();
  const Members MA = R.A->members(), MB = R.B->members();
  const Layer& A = *R.A;
  const Layer& OB = R.same ? *R.A : *R.B;
  if (R.gctx) {
    R.total += gpu_rows(R.gctx, *R.c, A, OB, GSJ_ENC_RELATE, R.same, R.distinct, false, 0.0, R.pat, p, nullptr, code, nullptr, n, &R.enc_s,
                        &R.wr_s);
    R.host_s += secs_since(th);
    return;
  }
  R.total += send_rows_acc(R, *R.c, n, [&](uint64_t i, FrameWriter& f) {
    const uint32_t cd = code[i], ct = gsj_de9im_transpose(cd);
    pair_rows(p[2 * i], p[2 * i + 1], MA, MB, R.same, R.distinct, [&](uint32_t ra, uint32_t rb, bool tr) {
      put_relate(f, R, A, ra, OB, rb, tr ? ct : cd);
    });
  });
  R.host_s += secs_since(th);
}
int relate_sink(void* u, const uint32_t* p, const double*, const uint32_t* code, uint64_t n) {
  RelateRun& R = *static_cast<RelateRun*>(u);
  R.out->push(p, nullptr, code, nullptr, n);
  return R.c->broken ? 1 : 0;
}

void relate_points_rows(RelateRun& R, const uint32_t* p, const uint8_t* wh, uint64_t n) {
  const auto th = Clock::now();
  const Members MB = R.B->members();
  if (R.gctx) {   // A points, B polygons
    R.total += gpu_rows(R.gctx, *R.c, *R.A, *R.B, GSJ_ENC_POINT_RELATE, false, false, R.swapped, 0.0, R.pat, p, nullptr, nullptr, wh, n,
                        &R.enc_s, &R.wr_s);
    R.host_s += secs_since(th);
    return;
  }
  R.total += send_rows_acc(R, *R.c, n, [&](uint64_t i, FrameWriter& f) {
    const uint32_t code = wh[i] == 2 ? kPtBoundary : kPtInterior;   // relate(point, polygon)
    MB.each(p[2 * i + 1], [&](uint32_t rb) {
      if (R.swapped) put_relate(f, R, *R.B, rb, *R.A, p[2 * i], gsj_de9im_transpose(code));
      else put_relate(f, R, *R.A, p[2 * i], *R.B, rb, code);
    });
  });
  R.host_s += secs_since(th);
}
int relate_points_sink(void* u, const uint32_t* p, const uint8_t* wh, uint64_t n) {
  RelateRun& R = *static_cast<RelateRun*>(u);
  R.out->push(p, nullptr, nullptr, wh, n);
  return R.c->broken ? 1 : 0;
}

void op_relate(Conn& c, const std::vector<std::string>& a) {
  if (a.size() < 4) throw std::runtime_error("RELATE needs layer_a, layer_b, pattern, self_pairs");
  auto A = get_layer(a[0]), B = get_layer(a[1]);
  const std::string pat = a[2];
  if (!pat.empty()) {
    if (pat.size() != 9) throw std::runtime_error("DE-9IM pattern must have 9 characters");
    for (char ch : pat)
      if (!strchr("TtFf*012", ch) || ch == 0) throw std::runtime_error("bad DE-9IM pattern character '" + std::string(1, ch) + "'");
  }
  const bool distinct = self_pairs_arg(a[3]);
  const bool same = A.get() == B.get();
  if (A->points() && B->points()) throw std::runtime_error("point x point relate is not supported");
  bool swapped = false;
  if (!A->points() && B->points()) { std::swap(A, B); swapped = true; }
  Lease lease(scratch_estimate(*A, *B), A->gpu_geoms <= kSmallGeoms);
  gsj_ctx* ctx = lease.get();
  c.u32(GSP_OK);
  c.streaming = true;
  gsj_join_opts o;
  gsj_join_opts_default(&o);
  o.cancel = &c.broken;
  o.refine_mode = g_cfg.refine_mode;
  const auto t0 = Clock::now();
  RelateRun R{&c, A.get(), B.get(), same, distinct, swapped, pat};
  const bool pipe = g_cfg.stream_batch > 0;
  if (pipe) o.batch_q = g_cfg.stream_batch;
  Streamer out(pipe, [&](const uint32_t* p, const double*, const uint32_t* code, const uint8_t* wh, uint64_t n) {
    if (R.A->points()) relate_points_rows(R, p, wh, n); else relate_rows(R, p, code, n);
  });
  R.out = &out;
  if (!pipe && g_cfg.gpu_encode && A->rs && B->rs) R.gctx = ctx;
  gsj_join_stats st{};
  if (A->points()) {
    const int rc = gsj_join_points(ctx, A->h, B->h, &o, relate_points_sink, &R, &st);
    out.finish();
    engine_status(c, ctx, rc, "relate");
  } else {
    gsj_refine_params rp;
    gsj_refine_params_default(&rp);
    rp.want_area = 0;
    rp.want_relate = 1;
    o.upper = same;
    const int rc = gsj_join(ctx, A->h, B->h, &rp, &o, relate_sink, &R, &st);
    out.finish();
    engine_status(c, ctx, rc, "relate");
  }
  const std::string stats = Json().str("kind", "relate").str("pattern", pat).u64("candidates", st.candidates).u64("gpu_hits", st.hits)
      .u64("rows", R.total).num("host_encode_send_s", R.host_s).num("host_encode_s", R.enc_s).num("host_write_s", R.wr_s).num("total_s", secs_since(t0)).done();
  if (!c.broken) c.end_stream(stats);
  logf("relate %s x %s: %s%s", a[0].c_str(), a[1].c_str(), stats.c_str(), c.broken ? " (client went away)" : "");
}

// ---- DWITHIN (op_dwithin, gpujoind.cu:391-484) ----------------------------------------------------------------------
double to_double(const std::string& s) {
  char* e;
  const double v = strtod(s.c_str(), &e);
  if (s.empty() || *e || !std::isfinite(v)) throw std::runtime_error("not a number: " + s);
  return v;
}

struct PairsRun {
  Conn* c;
  const Layer *A, *B, *LA, *LB;
  bool same, distinct, stats_only, swapped;
  uint64_t total = 0;
  double host_s = 0, enc_s = 0, wr_s = 0;
  Streamer* out = nullptr;
  gsj_ctx* gctx = nullptr;   // set: rows encoded on the device
};

void pairs_rows(PairsRun& P, const uint32_t* p, uint64_t n) {
  const auto th = Clock::now();
  const Members MA = P.A->members(), MB = P.B->members();
  if (P.A->points()) {   // (point, polygon parent) pairs
    if (P.stats_only) {
      for (uint64_t i = 0; i < n; i++) P.total += MB.count(p[2 * i + 1]);
    } else if (P.gctx) {
      P.total += gpu_rows(P.gctx, *P.c, *P.A, *P.B, GSJ_ENC_POINTS, false, false, P.swapped, kNaN, "", p, nullptr, nullptr, nullptr, n, &P.enc_s,
                          &P.wr_s);
    } else {
      P.total += send_rows_acc(P, *P.c, n, [&](uint64_t i, FrameWriter& f) {
        MB.each(p[2 * i + 1], [&](uint32_t rb) {
          uint32_t ra = p[2 * i];
          if (P.swapped) std::swap(ra, rb);
          f.id(P.LA->ids.data(ra), P.LA->ids.len(ra)); f.id(P.LB->ids.data(rb), P.LB->ids.len(rb)); f.f64(kNaN); f.row_done();
        });
      });
    }
  } else if (P.stats_only) {
    uint64_t t = 0;
#pragma omp parallel for num_threads(g_cfg.threads) reduction(+ : t)
    for (int64_t i = 0; i < (int64_t)n; i++) t += pair_row_count(p[2 * i], p[2 * i + 1], MA, MB, P.same, P.distinct);
    P.total += t;
  } else if (P.gctx) {
    P.total += gpu_rows(P.gctx, *P.c, *P.A, P.same ? *P.A : *P.B, GSJ_ENC_PAIRS, P.same, P.distinct, false, 0.0, "", p, nullptr, nullptr,
                        nullptr, n, &P.enc_s, &P.wr_s);
  } else {
    const Layer& A = *P.A;
    const Layer& OB = P.same ? *P.A : *P.B;
    P.total += send_rows_acc(P, *P.c, n, [&](uint64_t i, FrameWriter& f) {
      pair_rows(p[2 * i], p[2 * i + 1], MA, MB, P.same, P.distinct, [&](uint32_t ra, uint32_t rb, bool) {
        f.id(A.ids.data(ra), A.ids.len(ra)); f.id(OB.ids.data(rb), OB.ids.len(rb)); f.f64(kNaN); f.row_done();
      });
    });
  }
  P.host_s += secs_since(th);
}
int pairs_sink(void* u, const uint32_t* p, uint64_t n) {
  PairsRun& P = *static_cast<PairsRun*>(u);
  P.out->push(p, nullptr, nullptr, nullptr, n);
  return P.c->broken ? 1 : 0;
}

void op_dwithin(Conn& c, const std::vector<std::string>& a) {
  if (a.size() < 6) throw std::runtime_error("DWITHIN needs layer_a, layer_b, mode, dist_a, dist_b, self_pairs[, stats]");
  const bool stats_only = a.size() > 6 && a[6] == "stats";
  auto A = get_layer(a[0]), B = get_layer(a[1]);
  const std::string mode = a[2];
  const double da = to_double(a[3]), db = to_double(a[4]);
  const bool distinct = self_pairs_arg(a[5]);
  bool erode = false;
  double d = 0, ra = 0, rb = 0;
  if (mode == "dwithin") {
    if (da < 0) throw std::runtime_error("distance must be >= 0");
    d = da;
  } else if (mode == "buffer") {
    if (da <= 0 && db <= 0 && (da < 0 || db < 0)) { erode = true; ra = -da; rb = -db; }
    else if (da >= 0 && db >= 0) d = da + db;
    else throw std::runtime_error("buffers of opposite sign are not supported");
  } else {
    throw std::runtime_error("mode must be 'dwithin' or 'buffer'");
  }
  if (A->points() && B->points()) throw std::runtime_error("point x point distance joins are not supported");
  const bool same = A.get() == B.get();
  bool swapped = false;
  if (!A->points() && B->points()) { std::swap(A, B); std::swap(ra, rb); swapped = true; }
  if (A->points() && erode && ra > 0) throw std::runtime_error("a point layer cannot have a negative buffer");
  Lease lease(scratch_estimate(*A, *B), A->gpu_geoms <= kSmallGeoms);
  gsj_ctx* ctx = lease.get();
  c.u32(GSP_OK);
  c.streaming = true;
  gsj_join_opts o;
  gsj_join_opts_default(&o);
  o.cancel = &c.broken;
  o.refine_mode = g_cfg.refine_mode;
  const auto t0 = Clock::now();
  PairsRun P{&c, A.get(), B.get(), swapped ? B.get() : A.get(), swapped ? A.get() : B.get(), same, distinct, stats_only, swapped};
  // erosion keeps one batch: its pass-2 tiles work on the whole candidate set
  const bool pipe = !stats_only && !erode && g_cfg.stream_batch > 0;
  if (pipe) o.batch_q = g_cfg.stream_batch;
  Streamer out(pipe, [&](const uint32_t* p, const double*, const uint32_t*, const uint8_t*, uint64_t n) { pairs_rows(P, p, n); });
  P.out = &out;
  if (!pipe && g_cfg.gpu_encode && A->rs && B->rs) P.gctx = ctx;
  gsj_join_stats st{};
  if (A->points()) {
    const int rc = erode ? gsj_points_erode(ctx, A->h, B->h, rb, &o, pairs_sink, &P, &st) : gsj_points_dwithin(ctx, A->h, B->h, d, &o, pairs_sink, &P, &st);
    out.finish();
    engine_status(c, ctx, rc, "dwithin");
  } else {
    o.upper = same;
    if (erode) {
      std::vector<uint8_t> need;   // a geometry's pair with itself matters only for groups of identical rows
      if (same && distinct) {
        need.assign(A->n_distinct, 0);
        if (A->deduped) for (uint64_t g = 0; g < A->n_distinct; g++) need[g] = A->moff[g + 1] - A->moff[g] > 1;
      }
      const int rc = gsj_erode(ctx, A->h, B->h, ra, rb, same, need.empty() ? nullptr : need.data(), &o, pairs_sink, &P, &st);
      out.finish();
      engine_status(c, ctx, rc, "dwithin");
    } else {
      const int rc = gsj_dwithin(ctx, A->h, B->h, d, same, &o, pairs_sink, &P, &st);
      out.finish();
      engine_status(c, ctx, rc, "dwithin");
    }
  }
  const std::string stats = Json().str("kind", erode ? "buffer_intersects" : "dwithin").num("distance_m", d).num("erode_a_m", swapped ? rb : ra)
      .num("erode_b_m", swapped ? ra : rb).u64("candidates", st.candidates).u64("tested", st.candidates).u64("gpu_hits", st.hits)
      .u64("rows", P.total).u64("heavy", st.heavy).num("traverse_ms", st.traverse_ms).num("refine_ms", st.refine_ms)
      .num("compact_ms", st.compact_ms).num("d2h_ms", st.copy_ms).num("host_encode_send_s", P.host_s).num("host_encode_s", P.enc_s).num("host_write_s", P.wr_s).num("total_s", secs_since(t0))
      .boolean("stats_only", stats_only).done();
  if (!c.broken) c.end_stream(stats);
  logf("dwithin %s x %s %s %s %s: %s%s", a[0].c_str(), a[1].c_str(), mode.c_str(), a[3].c_str(), a[4].c_str(), stats.c_str(),
       c.broken ? " (client went away)" : "");
}

// ---- JSON ops -----------------------------------------------------------------------------------------------------
std::string layer_names() {
  std::lock_guard<std::mutex> r(g_reg);
  std::string ls = "[";
  bool first = true;
  for (auto& kv : g_layers) { if (!first) ls += ","; first = false; ls += jquote(kv.first); }
  return ls + "]";
}

std::string op_status() {   // gpujoind.cu:486-494 (+ the worker pool)
  char name[256] = {0};
  int ma = 0, mi = 0;
  uint64_t fr = 0, tot = 0;
  const int rc = gsj_device_query(g_cfg.device, name, sizeof name, &ma, &mi, &fr, &tot);
  if (rc) throw std::runtime_error("no usable CUDA device " + std::to_string(g_cfg.device));
  int busy = 0;
  uint64_t queued = 0, used = 0, budget = 0;
  g_pool_small.counts(&busy, &queued, &used, &budget);
  g_pool_large.counts(&busy, &queued, &used, &budget);
  return Json().str("device", name).str("cc", std::to_string(ma) + "." + std::to_string(mi)).num("mem_total_mb", tot / 1048576.0)
      .num("mem_free_mb", fr / 1048576.0).key("layers").raw(layer_names()).u64("workers", (uint64_t)g_cfg.workers)
      .u64("busy", (uint64_t)busy).u64("queued", queued).num("scratch_used_mb", used / 1048576.0).num("scratch_budget_mb", budget / 1048576.0)
      .str("refine", g_cfg.refine_mode == GSJ_REFINE_PLAIN ? "plain" : "filtered").done();
}

std::string op_list() {
  std::lock_guard<std::mutex> r(g_reg);
  std::string s = "[";
  bool first = true;
  for (auto& kv : g_layers) { if (!first) s += ","; first = false; s += kv.second->json(); }
  return s + "]";
}

int to_int(const std::string& s, int dflt) {
  if (s.empty()) return dflt;
  char* e;
  const long v = strtol(s.c_str(), &e, 10);
  if (*e) throw std::runtime_error("not an integer: " + s);
  return (int)v;
}
bool to_bool(const std::string& s, bool dflt) {
  if (s.empty()) return dflt;
  return s == "1" || s == "t" || s == "true" || s == "on";
}

bool token_ok(const std::string& tok) {   // constant time in the token's length (gpujoind.cu:527-533)
  unsigned diff = tok.size() != g_cfg.token.size();
  for (size_t i = 0; i < g_cfg.token.size(); i++)
    diff |= (unsigned)(uint8_t)g_cfg.token[i] ^ (unsigned)(uint8_t)(i < tok.size() ? tok[i] : 0);
  return diff == 0;
}

void handle(int fd) {
  Conn c{fd};
  try {
    uint32_t hdr[3];
    if (!c.read_full(hdr, 12) || hdr[0] != GSP_MAGIC || hdr[2] > GSP_MAX_ARGS) { close(fd); return; }
    std::vector<std::string> args(hdr[2]);
    for (auto& s : args) {
      uint32_t l;
      if (!c.read_full(&l, 4) || l > GSP_MAX_ARG_BYTES) { close(fd); return; }
      s.resize(l);
      if (l && !c.read_full(&s[0], l)) { close(fd); return; }
    }
    if (!token_ok(args.empty() ? std::string() : args[0])) {
      logf("rejected request: bad token");
      c.error("authentication failed");
      close(fd);
      return;
    }
    if (!args.empty()) args.erase(args.begin());
    switch (hdr[1]) {
      case GSP_OP_LOAD: {
        if (args.size() < 7) throw std::runtime_error("LOAD needs 7 args");
        // args: layer, table (a file), id_col, geom_col (the file's two columns), filter, subdivide, dedup
        if (!args[4].empty()) throw std::runtime_error("a row filter needs PostgreSQL: filter the rows when writing the COPY file");
        c.ok_json(build_layer(args[0], resolve_path(args[1]), to_int(args[5], 0), to_bool(args[6], true)));
        break;
      }
      case GSP_OP_LOAD_QUERY:
        throw std::runtime_error("LOAD_QUERY runs SQL over libpq, which this daemon does not link: write the query's rows with "
                                 "COPY (SELECT id::text, geom ...) TO 'file' (FORMAT binary) and LOAD the file");
      case GSP_OP_DROP: {
        if (args.empty()) throw std::runtime_error("DROP needs layer");
        std::shared_ptr<Layer> old;
        {
          std::lock_guard<std::mutex> g(g_reg);
          auto it = g_layers.find(args[0]);
          if (it != g_layers.end()) { old = it->second; g_layers.erase(it); }
        }
        if (old && !g_cfg.snapshot_dir.empty()) remove(snapshot_path(args[0]).c_str());   // not restored any more
        c.ok_json(old ? "true" : "false");
        break;
      }
      case GSP_OP_LIST: c.ok_json(op_list()); break;
      case GSP_OP_STATUS: c.ok_json(op_status()); break;
      case GSP_OP_JOIN: op_join(c, args); break;
      case GSP_OP_CLUSTER: op_cluster(c, args); break;
      case GSP_OP_RELATE: op_relate(c, args); break;
      case GSP_OP_DWITHIN: op_dwithin(c, args); break;
      default: c.error("unknown op");
    }
  } catch (const std::exception& e) {
    logf("error: %s", e.what());
    if (c.streaming) { c.u32(GSP_FRAME_ERR); c.str(e.what()); }
    else c.error(e.what());
  }
  close(fd);
}

// ---- listeners ----------------------------------------------------------------------------------------------------
int listen_unix(const std::string& path) {
  const int fd = socket(AF_UNIX, SOCK_STREAM, 0);
  sockaddr_un a{};
  a.sun_family = AF_UNIX;
  if (path.size() >= sizeof(a.sun_path)) { fprintf(stderr, "socket path too long\n"); return -1; }
  strncpy(a.sun_path, path.c_str(), sizeof(a.sun_path) - 1);
  unlink(path.c_str());
  if (bind(fd, (sockaddr*)&a, sizeof a) || listen(fd, 64)) { perror(("unix socket " + path).c_str()); close(fd); return -1; }
  chmod(path.c_str(), 0666);
  return fd;
}
int listen_tcp(const std::string& hp) {
  const auto pos = hp.rfind(':');
  if (pos == std::string::npos) { fprintf(stderr, "--tcp wants HOST:PORT\n"); return -1; }
  const std::string host = hp.substr(0, pos);
  const int port = atoi(hp.c_str() + pos + 1);
  const int fd = socket(AF_INET, SOCK_STREAM, 0), one = 1;
  setsockopt(fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof one);
  sockaddr_in a{};
  a.sin_family = AF_INET;
  a.sin_port = htons((uint16_t)port);
  if (inet_pton(AF_INET, host.c_str(), &a.sin_addr) != 1) { fprintf(stderr, "bad tcp address %s\n", hp.c_str()); close(fd); return -1; }
  if (bind(fd, (sockaddr*)&a, sizeof a) || listen(fd, 64)) { perror(("tcp " + hp).c_str()); close(fd); return -1; }
  return fd;
}

void on_signal(int) { g_stop = true; }

const char* kUsage =
    "usage: gsjd [--socket PATH] [--tcp HOST:PORT] [--token-file FILE] [--data-dir DIR] [--device N] [--workers N]\n"
    "            [--threads N] [--mem-budget-gb G] [--refine plain|filtered] [--stream-batch N] [--gpu-encode 0|1]\n"
    "            [--snapshot-dir DIR (prepared layers saved after LOAD, restored at start-up)]\n"
    "            [--tune 0|1 (refinement autotuner on each LOADed polygon layer of >= 100k geometries)]\n"
    "            [--conninfo STR (accepted, unused: layers load from files)]\n";

}  // namespace
}  // namespace gsjd

extern "C" int gsjd_main(int argc, char** argv) {
  using namespace gsjd;
  // a server: load every kernel at context creation, not at its first launch in the middle of a request (unless
  // the caller chose a loading mode)
  setenv("CUDA_MODULE_LOADING", "EAGER", 0);
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    const bool has = i + 1 < argc;
    if (a == "--socket" && has) g_cfg.socket = argv[++i];
    else if (a == "--tcp" && has) g_cfg.tcp = argv[++i];
    else if (a == "--data-dir" && has) g_cfg.data_dir = argv[++i];
    else if (a == "--device" && has) g_cfg.device = atoi(argv[++i]);
    else if (a == "--workers" && has) g_cfg.workers = std::max(1, atoi(argv[++i]));
    else if (a == "--threads" && has) g_cfg.threads = std::max(1, atoi(argv[++i]));
    else if (a == "--mem-budget-gb" && has) g_cfg.mem_budget_gb = atof(argv[++i]);
    else if (a == "--stream-batch" && has) g_cfg.stream_batch = (uint32_t)std::max(0, atoi(argv[++i]));
    else if (a == "--gpu-encode" && has) g_cfg.gpu_encode = atoi(argv[++i]) != 0;
    else if (a == "--snapshot-dir" && has) g_cfg.snapshot_dir = argv[++i];
    else if (a == "--tune" && has) g_cfg.tune = atoi(argv[++i]) != 0;
    else if (a == "--refine" && has) {
      const std::string m = argv[++i];
      if (m != "plain" && m != "filtered") { fputs("--refine plain|filtered\n", stderr); return 1; }
      g_cfg.refine_mode = m == "plain" ? GSJ_REFINE_PLAIN : GSJ_REFINE_FILTERED;
    }
    else if (a == "--conninfo" && has) ++i;
    else if (a == "--token-file" && has) {
      std::ifstream tf(argv[++i]);
      std::getline(tf, g_cfg.token);
      if (g_cfg.token.empty()) { fprintf(stderr, "empty token file\n"); return 1; }
    } else {
      fputs(kUsage, stderr);
      return 1;
    }
  }
  if (!g_cfg.tcp.empty() && g_cfg.token.empty()) { fprintf(stderr, "--tcp requires --token-file\n"); return 1; }
  signal(SIGPIPE, SIG_IGN);
  struct sigaction sa{};
  sa.sa_handler = on_signal;   // no SA_RESTART: poll() returns and the loop sees the flag
  sigaction(SIGTERM, &sa, nullptr);
  sigaction(SIGINT, &sa, nullptr);
  g_encode.start(std::max(0, g_cfg.threads - 1));
  g_pool_small.prewarm();   // before the socket exists: a client that can connect finds the contexts ready
  g_pool_large.prewarm();
  restore_snapshots();
  std::vector<pollfd> fds;
  const int u = listen_unix(g_cfg.socket);
  if (u < 0) return 1;
  fds.push_back({u, POLLIN, 0});
  logf("gsjd listening on unix:%s (device %d, %d workers, data dir %s)", g_cfg.socket.c_str(), g_cfg.device, g_cfg.workers, g_cfg.data_dir.c_str());
  if (!g_cfg.tcp.empty()) {
    const int t = listen_tcp(g_cfg.tcp);
    if (t < 0) return 1;
    fds.push_back({t, POLLIN, 0});
    logf("listening on tcp:%s", g_cfg.tcp.c_str());
  }
  while (!g_stop) {
    if (poll(fds.data(), fds.size(), 500) < 0) {
      if (errno == EINTR) continue;
      perror("poll");
      return 1;
    }
    for (auto& f : fds)
      if (f.revents & POLLIN) {
        const int cfd = accept(f.fd, nullptr, nullptr);
        if (cfd < 0) continue;
        const int one = 1;
        setsockopt(cfd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof one);
        std::thread(handle, cfd).detach();
      }
  }
  for (auto& f : fds) close(f.fd);
  unlink(g_cfg.socket.c_str());
  logf("gsjd stopped");
  return 0;
}
