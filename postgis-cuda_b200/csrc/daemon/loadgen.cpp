// gsjd_loadgen: load generator for the daemon. Replays a schedule of requests (arrival time, op, args) against a
// gsjd (or gpujoind) socket, one connection per request started at its arrival time (open loop), reads every
// result stream to its end, and prints a JSON summary of the latencies (arrival to end of stream, so time spent
// queueing in the daemon counts) and row counts. With --closed N the arrival times are ignored: N clients each send
// the schedule's requests in turn (shared order), the next as soon as the previous result stream ended, for
// --duration seconds, and the summary adds the served rows per second (the daemon at saturation).
//
//   gsjd_loadgen --socket PATH [--token TOKEN] --schedule FILE [--warmup N] [--detail FILE] [--closed N --duration S]
//
// --detail writes one TSV line per request: index, op, first argument (the query layer), arrival s, latency ms
// (-1 on error), rows, first-row ms (arrival to the first frame header), and the daemon's stats JSON.
//
// Schedule lines: <arrival seconds> TAB <op name> TAB <arg> TAB <arg> ...   (op: JOIN RELATE DWITHIN CLUSTER)
#include <sys/socket.h>
#include <sys/un.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/gsp_protocol.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  double t = 0;
  uint32_t op = 0;
  std::string name;
  std::vector<std::string> args;
};
struct Result {
  double latency_s = -1, first_s = -1;
  uint64_t rows = 0;
  std::string stats;
  bool ok = false;
  std::string err;
};

class Sock {
 public:
  explicit Sock(int fd) : fd_(fd) {}
  ~Sock() { if (fd_ >= 0) close(fd_); }
  bool send_all(const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    while (n) {
      const ssize_t r = ::send(fd_, c, n, MSG_NOSIGNAL);
      if (r <= 0) return false;
      c += r; n -= (size_t)r;
    }
    return true;
  }
  bool read(void* p, size_t n) {   // buffered; the common case is a copy out of the buffer
    if (len_ - pos_ >= n) { std::memcpy(p, buf_ + pos_, n); pos_ += n; return true; }
    return read_slow(p, n);
  }
  bool skip(size_t n) {
    if (len_ - pos_ >= n) { pos_ += n; return true; }
    return skip_slow(n);
  }
  bool read_slow(void* p, size_t n) {
    char* o = static_cast<char*>(p);
    while (n) {
      if (pos_ == len_) {
        const ssize_t r = ::read(fd_, buf_, sizeof buf_);
        if (r <= 0) return false;
        pos_ = 0; len_ = (size_t)r;
      }
      const size_t k = std::min(n, len_ - pos_);
      std::memcpy(o, buf_ + pos_, k);
      pos_ += k; o += k; n -= k;
    }
    return true;
  }
  bool skip_slow(size_t n) {
    while (n) {
      if (pos_ == len_) {
        const ssize_t r = ::read(fd_, buf_, sizeof buf_);
        if (r <= 0) return false;
        pos_ = 0; len_ = (size_t)r;
      }
      const size_t k = std::min(n, len_ - pos_);
      pos_ += k; n -= k;
    }
    return true;
  }
  bool u32(uint32_t& v) { return read(&v, 4); }
  bool str(std::string& s) {
    uint32_t l;
    if (!u32(l)) return false;
    s.resize(l);
    return !l || read(&s[0], l);
  }

 private:
  int fd_;
  char buf_[1 << 20];
  size_t pos_ = 0, len_ = 0;
};

std::string g_socket, g_token;

int connect_unix() {
  const int fd = socket(AF_UNIX, SOCK_STREAM, 0);
  sockaddr_un a{};
  a.sun_family = AF_UNIX;
  strncpy(a.sun_path, g_socket.c_str(), sizeof(a.sun_path) - 1);
  if (connect(fd, (sockaddr*)&a, sizeof a)) { close(fd); return -1; }
  return fd;
}

Result run(const Req& q, Clock::time_point arrival) {
  Result res;
  const int fd = connect_unix();
  if (fd < 0) { res.err = "connect failed"; return res; }
  Sock s(fd);
  std::string msg;
  auto put32 = [&](uint32_t v) { msg.append(reinterpret_cast<const char*>(&v), 4); };
  put32(GSP_MAGIC); put32(q.op); put32((uint32_t)q.args.size() + 1);
  put32((uint32_t)g_token.size()); msg += g_token;
  for (auto& a : q.args) { put32((uint32_t)a.size()); msg += a; }
  if (!s.send_all(msg.data(), msg.size())) { res.err = "send failed"; return res; }
  uint32_t st;
  if (!s.u32(st)) { res.err = "no response"; return res; }
  if (st != GSP_OK) { s.str(res.err); return res; }
  for (;;) {
    uint32_t n;
    if (!s.u32(n)) { res.err = "stream cut"; return res; }
    if (res.first_s < 0) res.first_s = std::chrono::duration<double>(Clock::now() - arrival).count();
    if (n == GSP_FRAME_ERR) { s.str(res.err); return res; }
    if (n == 0) break;
    for (uint32_t i = 0; i < n; i++) {
      uint16_t l;
      if (!s.read(&l, 2) || !s.skip(l)) { res.err = "stream cut"; return res; }
      if (q.op == GSP_OP_CLUSTER) { if (!s.skip(4)) { res.err = "stream cut"; return res; } continue; }
      if (!s.read(&l, 2) || !s.skip(l) || !s.skip(q.op == GSP_OP_RELATE ? 9 : 8)) { res.err = "stream cut"; return res; }
    }
    res.rows += n;
  }
  if (!s.str(res.stats)) { res.err = "no stats"; return res; }
  res.latency_s = std::chrono::duration<double>(Clock::now() - arrival).count();
  res.ok = true;
  return res;
}

double pct(std::vector<double> v, double p) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  const double k = p / 100.0 * (double)(v.size() - 1);
  const size_t i = (size_t)k;
  const double f = k - (double)i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

uint32_t op_code(const std::string& s) {
  static const std::map<std::string, uint32_t> m = {{"JOIN", GSP_OP_JOIN}, {"RELATE", GSP_OP_RELATE}, {"DWITHIN", GSP_OP_DWITHIN},
                                                   {"CLUSTER", GSP_OP_CLUSTER}};
  auto it = m.find(s);
  return it == m.end() ? 0 : it->second;
}

// closed loop: N clients, each starting the next request of the shared order when its previous one ended
std::string closed_loop(const std::vector<Req>& reqs, int clients, double duration) {
  std::atomic<uint64_t> next{0};
  std::mutex mu;
  std::vector<double> lat;
  uint64_t rows = 0, done = 0, errors = 0;
  std::string first_err;
  const auto t0 = Clock::now();
  const auto until = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(duration));
  std::vector<std::thread> th;
  for (int c = 0; c < clients; c++)
    th.emplace_back([&] {
      while (Clock::now() < until) {
        const Req& q = reqs[next.fetch_add(1) % reqs.size()];
        const Result r = run(q, Clock::now());
        std::lock_guard<std::mutex> g(mu);
        if (!r.ok) { errors++; if (first_err.empty()) first_err = r.err; continue; }
        lat.push_back(r.latency_s);
        rows += r.rows;
        done++;
      }
    });
  for (auto& t : th) t.join();
  const double span = std::chrono::duration<double>(Clock::now() - t0).count();
  char b[512];
  snprintf(b, sizeof b, "{\"mode\":\"closed\",\"clients\":%d,\"requests\":%llu,\"errors\":%llu,\"rows\":%llu,\"span_s\":%.6g,"
           "\"rows_per_s\":%.6g,\"requests_per_s\":%.6g,\"p50_ms\":%.6g,\"p99_ms\":%.6g", clients, (unsigned long long)done,
           (unsigned long long)errors, (unsigned long long)rows, span, rows / span, done / span, 1e3 * pct(lat, 50), 1e3 * pct(lat, 99));
  std::string js = b;
  if (!first_err.empty()) {
    std::string e;
    for (char ch : first_err) { if (ch == '"' || ch == '\\') e += '\\'; if ((unsigned char)ch >= 0x20) e += ch; }
    js += ",\"first_error\":\"" + e + "\"";
  }
  return js + "}";
}

}  // namespace

int main(int argc, char** argv) {
  std::string sched, detail;
  size_t warmup = 0;
  int closed = 0;
  double duration = 10.0;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--socket" && i + 1 < argc) g_socket = argv[++i];
    else if (a == "--token" && i + 1 < argc) g_token = argv[++i];
    else if (a == "--schedule" && i + 1 < argc) sched = argv[++i];
    else if (a == "--warmup" && i + 1 < argc) warmup = (size_t)atol(argv[++i]);
    else if (a == "--detail" && i + 1 < argc) detail = argv[++i];
    else if (a == "--closed" && i + 1 < argc) closed = atoi(argv[++i]);
    else if (a == "--duration" && i + 1 < argc) duration = atof(argv[++i]);
    else {
      fprintf(stderr, "usage: gsjd_loadgen --socket PATH [--token T] --schedule FILE [--warmup N] [--detail FILE] [--closed N --duration S]\n");
      return 2;
    }
  }
  std::ifstream f(sched);
  if (!f) { fprintf(stderr, "cannot read schedule %s\n", sched.c_str()); return 2; }
  std::vector<Req> reqs;
  for (std::string line; std::getline(f, line);) {
    if (line.empty() || line[0] == '#') continue;
    std::vector<std::string> col;
    std::stringstream ss(line);
    for (std::string c; std::getline(ss, c, '\t');) col.push_back(c);
    if (col.size() < 2) continue;
    Req q;
    q.t = atof(col[0].c_str());
    q.name = col[1];
    q.op = op_code(col[1]);
    if (!q.op) { fprintf(stderr, "unknown op %s\n", col[1].c_str()); return 2; }
    q.args.assign(col.begin() + 2, col.end());
    reqs.push_back(q);
  }
  if (reqs.empty()) { fprintf(stderr, "empty schedule\n"); return 2; }
  if (closed > 0) {
    const std::string js = closed_loop(reqs, closed, duration);
    puts(js.c_str());
    return js.find("\"errors\":0,") == std::string::npos ? 1 : 0;
  }
  std::vector<Result> res(reqs.size());
  std::vector<std::thread> th;
  th.reserve(reqs.size());
  const auto t0 = Clock::now() + std::chrono::milliseconds(50);
  for (size_t i = 0; i < reqs.size(); i++) {
    const auto at = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(reqs[i].t));
    std::this_thread::sleep_until(at);
    th.emplace_back([&, i, at] { res[i] = run(reqs[i], at); });
  }
  for (auto& t : th) t.join();
  const double span = std::chrono::duration<double>(Clock::now() - t0).count();
  if (!detail.empty()) {
    FILE* df = fopen(detail.c_str(), "w");
    if (!df) { fprintf(stderr, "cannot write %s\n", detail.c_str()); return 2; }
    for (size_t i = 0; i < res.size(); i++)
      fprintf(df, "%zu\t%s\t%s\t%.6f\t%.4f\t%llu\t%.4f\t%s\n", i, reqs[i].name.c_str(), reqs[i].args.empty() ? "" : reqs[i].args[0].c_str(),
              reqs[i].t, res[i].ok ? 1e3 * res[i].latency_s : -1.0, (unsigned long long)res[i].rows, 1e3 * res[i].first_s,
              res[i].stats.c_str());
    fclose(df);
  }
  std::vector<double> lat;
  std::map<std::string, std::vector<double>> per;
  uint64_t rows = 0, errors = 0;
  std::string first_err;
  for (size_t i = 0; i < res.size(); i++) {
    if (!res[i].ok) { errors++; if (first_err.empty()) first_err = res[i].err; continue; }
    if (i < warmup) continue;
    lat.push_back(res[i].latency_s);
    per[reqs[i].name].push_back(res[i].latency_s);
    rows += res[i].rows;
  }
  std::string js = "{\"requests\":" + std::to_string(reqs.size()) + ",\"measured\":" + std::to_string(lat.size()) +
                   ",\"errors\":" + std::to_string(errors) + ",\"rows\":" + std::to_string(rows);
  char b[512];
  snprintf(b, sizeof b, ",\"span_s\":%.6g,\"p50_ms\":%.6g,\"p90_ms\":%.6g,\"p99_ms\":%.6g,\"max_ms\":%.6g", span, 1e3 * pct(lat, 50),
           1e3 * pct(lat, 90), 1e3 * pct(lat, 99), 1e3 * pct(lat, 100));
  js += b;
  js += ",\"by_op\":{";
  bool first = true;
  for (auto& kv : per) {
    snprintf(b, sizeof b, "%s\"%s\":{\"n\":%zu,\"p50_ms\":%.6g,\"p99_ms\":%.6g}", first ? "" : ",", kv.first.c_str(), kv.second.size(),
             1e3 * pct(kv.second, 50), 1e3 * pct(kv.second, 99));
    js += b;
    first = false;
  }
  js += "}";
  if (!first_err.empty()) {
    std::string e;
    for (char c : first_err) { if (c == '"' || c == '\\') e += '\\'; if ((unsigned char)c >= 0x20) e += c; }
    js += ",\"first_error\":\"" + e + "\"";
  }
  js += "}";
  puts(js.c_str());
  return errors ? 1 : 0;
}
