// Network front end and write-ahead log of the served path (rg_frontend_*,
// rg_wal_* in include/risgraph_b200.h).
//
// The reference's served driver (src/all_inc_rpc.cpp) receives
// ClientUpdateRequest structs from remote clients (core/rpc.hpp:19-32), one
// receiving fiber per client, and answers each update with a
// ClientUpdateResponse carrying the label version (:34-38).  The first
// connection opens with clock-synchronisation requests that are answered with
// {0, 0} and give the mean offset between the client's clock and the server's
// (src/all_inc_rpc.cpp:277-290).  With its WAL enabled, each update is appended
// to the current 4 KB block and is applied only when that block is on disk;
// one writer swaps the filling block for the syncing one and writes it, so all
// updates that arrived while the previous block was being written share one
// write (group commit, :306-335, :572-589).
//
// Here the structs travel over TCP in the reference's byte layout.  One reader
// thread per connection parses requests; updates go to the GPU server
// (rg_server_submit) directly or, with the WAL, through a writer thread that
// submits each block's updates, in log order, once pwrite + fdatasync of the
// block returned.  One completion thread drains the server
// (rg_server_poll_wait) and sends the responses of each connection in request
// order.
#include <arpa/inet.h>
#include <fcntl.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <poll.h>
#include <sys/socket.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "risgraph_b200.h"

static_assert(sizeof(rg_client_update_request) == 40, "ClientUpdateRequest is 40 bytes on x86-64");
static_assert(sizeof(rg_client_update_response) == 16, "ClientUpdateResponse is 16 bytes on x86-64");
static_assert(sizeof(rg_wal_record) == 32, "a WAL record is 32 bytes");

namespace rg {
void set_error(const std::string &msg);
int server_check(rg_server *s, const rg_request &r);
}  // namespace rg

namespace {

constexpr size_t WAL_BLOCK = 4096;
constexpr size_t WAL_RECS = (WAL_BLOCK - 16) / sizeof(rg_wal_record);  // 127
constexpr uint64_t SEQ_BITS = 40, SEQ_MASK = (1ull << SEQ_BITS) - 1;
constexpr uint32_t REQ_ADD = 0, REQ_DEL = 1, REQ_END = 2;

struct WalBlock {
  uint64_t version, n;
  rg_wal_record rec[WAL_RECS];
  char pad[WAL_BLOCK - 16 - WAL_RECS * sizeof(rg_wal_record)];
};
static_assert(sizeof(WalBlock) == WAL_BLOCK, "one WAL block is 4 KB");

int64_t realtime_ns() {
  timespec ts;
  clock_gettime(CLOCK_REALTIME, &ts);
  return (int64_t)ts.tv_sec * 1000000000ll + ts.tv_nsec;
}

bool read_full(int fd, void *p, size_t n) {
  char *c = static_cast<char *>(p);
  while (n) {
    ssize_t r = recv(fd, c, n, 0);
    if (r <= 0) {
      if (r < 0 && errno == EINTR) continue;
      return false;
    }
    c += r;
    n -= (size_t)r;
  }
  return true;
}

bool write_full(int fd, const void *p, size_t n) {
  const char *c = static_cast<const char *>(p);
  while (n) {
    ssize_t r = send(fd, c, n, MSG_NOSIGNAL);
    if (r <= 0) {
      if (r < 0 && errno == EINTR) continue;
      return false;
    }
    c += r;
    n -= (size_t)r;
  }
  return true;
}

// One request awaiting its response on a connection.
struct Slot {
  uint32_t client_id;
  bool done, end;
  uint64_t version;
  int64_t t_req;  // request_time on the server's clock
};

struct Conn {
  int fd = -1;
  uint32_t index = 0;
  std::mutex mu;  // slots, head, last_version, the socket's write side
  std::deque<Slot> slots;
  uint64_t head = 0;  // sequence number of slots.front()
  uint64_t last_version = 0;
  bool broken = false;
  std::thread reader;
};

}  // namespace

struct rg_frontend {
  rg_server *srv = nullptr;
  uint32_t instance = 0;
  int lfd = -1;
  uint16_t port = 0;
  std::atomic<bool> stop_accept{false}, stop_completer{false};
  std::thread acceptor, completer, waler;
  std::mutex cmu;  // conns
  std::vector<std::shared_ptr<Conn>> conns;
  std::atomic<int64_t> in_flight{0};
  // clock synchronisation (first connection only)
  uint32_t sync_left = 0;
  int64_t offset_sum = 0;
  uint64_t sync_n = 0;
  std::atomic<int64_t> offset{0};
  // write-ahead log
  int wal_fd = -1;
  std::mutex wmu;
  std::condition_variable wcv;
  bool wal_stop = false;
  WalBlock *writing = nullptr, *syncing = nullptr;
  struct Pending {
    uint64_t version;
    rg_request req;
  };
  std::deque<Pending> pend;
  // statistics
  std::mutex smu;
  std::vector<uint64_t> lat;
  std::atomic<uint64_t> n_conn{0}, n_req{0}, n_upd{0}, n_sync{0}, n_blocks{0}, n_failed{0};
};

namespace {

// Send the responses at the head of a connection whose requests completed
// (caller holds c.mu).
void flush_conn(rg_frontend *f, Conn &c) {
  std::vector<rg_client_update_response> out;
  const int64_t now = realtime_ns();
  std::vector<uint64_t> lat;
  while (!c.slots.empty() && c.slots.front().done) {
    Slot &s = c.slots.front();
    if (s.end) s.version = c.last_version;
    out.push_back(rg_client_update_response{s.client_id, 0, s.version});
    if (!s.end) lat.push_back((uint64_t)std::max<int64_t>(0, now - s.t_req));
    c.slots.pop_front();
    c.head++;
  }
  if (!out.empty() && !c.broken && !write_full(c.fd, out.data(), out.size() * sizeof(out[0]))) c.broken = true;
  if (!lat.empty()) {
    std::lock_guard<std::mutex> lk(f->smu);
    f->lat.insert(f->lat.end(), lat.begin(), lat.end());
  }
}

std::shared_ptr<Conn> conn_of(rg_frontend *f, uint64_t tag) {
  std::lock_guard<std::mutex> lk(f->cmu);
  const uint64_t ci = tag >> SEQ_BITS;
  return ci < f->conns.size() ? f->conns[ci] : nullptr;
}

// Mark the request `tag` answered with `version` and send what is ready.
void complete(rg_frontend *f, uint64_t tag, uint64_t version) {
  std::shared_ptr<Conn> c = conn_of(f, tag);
  if (c) {
    std::lock_guard<std::mutex> lk(c->mu);
    const uint64_t seq = tag & SEQ_MASK;
    if (seq >= c->head && seq - c->head < c->slots.size()) {
      Slot &s = c->slots[seq - c->head];
      s.done = true;
      s.version = version;
      if (version != ~0ull) c->last_version = std::max(c->last_version, version);
      flush_conn(f, *c);
    }
  }
  f->in_flight--;
}

// A request the server refuses (a vertex id out of range, a weight too
// large) is answered at once with version ~0 (the reference would throw).
void refuse(rg_frontend *f, const rg_request &r) {
  f->n_failed++;
  complete(f, r.tag, ~0ull);
}

// Submit in order; when the server refuses the batch, submit one by one so
// that only the bad requests are refused.
void submit(rg_frontend *f, const rg_request *r, uint64_t n) {
  if (!n || rg_server_submit(f->srv, r, n) == RG_OK) return;
  for (uint64_t i = 0; i < n; i++)
    if (rg_server_submit(f->srv, &r[i], 1) != RG_OK) refuse(f, r[i]);
}

// One update on its way to the server (with the WAL: once its block is durable).
void forward(rg_frontend *f, const rg_request &r, const rg_client_update_request &q) {
  if (rg::server_check(f->srv, r) != RG_OK) {  // never logged, never applied
    refuse(f, r);
    return;
  }
  if (f->wal_fd < 0) {
    submit(f, &r, 1);
    return;
  }
  std::unique_lock<std::mutex> lk(f->wmu);
  f->wcv.wait(lk, [&] { return f->writing->n < WAL_RECS || f->wal_stop; });
  f->writing->rec[f->writing->n++] = rg_wal_record{q.type, q.client_id, q.src, q.dst, q.data};
  f->pend.push_back(rg_frontend::Pending{f->writing->version, r});
  lk.unlock();
  f->wcv.notify_all();
}

void reader_main(rg_frontend *f, std::shared_ptr<Conn> c, bool sync_conn) {
  rg_client_update_request q;
  while (read_full(c->fd, &q, sizeof(q))) {
    f->n_req++;
    if (sync_conn && f->sync_left) {
      // clock synchronisation: offset = server clock - client clock, answered {0, 0}
      f->sync_left--;
      f->offset_sum += realtime_ns() - q.request_time_ns;
      f->sync_n++;
      f->offset.store(f->offset_sum / (int64_t)f->sync_n);
      f->n_sync++;
      rg_client_update_response z{0, 0, 0};
      std::lock_guard<std::mutex> lk(c->mu);
      if (!write_full(c->fd, &z, sizeof(z))) break;
      continue;
    }
    if (q.type > REQ_END) break;  // not a request of this protocol: drop the connection
    uint64_t seq;
    {
      std::lock_guard<std::mutex> lk(c->mu);
      seq = c->head + c->slots.size();
      const bool end = q.type == REQ_END;
      c->slots.push_back(Slot{q.client_id, end, end, 0, q.request_time_ns + f->offset.load()});
      if (end) {  // answered after this connection's earlier requests
        flush_conn(f, *c);
        continue;
      }
    }
    f->n_upd++;
    rg_request r{f->instance, q.type, q.src, q.dst, q.data, ((uint64_t)c->index << SEQ_BITS) | (seq & SEQ_MASK)};
    f->in_flight++;
    forward(f, r, q);
  }
}

void acceptor_main(rg_frontend *f) {
  bool first = true;
  while (!f->stop_accept.load()) {
    pollfd p{f->lfd, POLLIN, 0};
    if (poll(&p, 1, 50) <= 0 || !(p.revents & POLLIN)) continue;
    int fd = accept(f->lfd, nullptr, nullptr);
    if (fd < 0) continue;
    int one = 1;
    setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof(one));
    auto c = std::make_shared<Conn>();
    c->fd = fd;
    {
      std::lock_guard<std::mutex> lk(f->cmu);
      c->index = (uint32_t)f->conns.size();
      f->conns.push_back(c);
    }
    f->n_conn++;
    c->reader = std::thread(reader_main, f, c, first);
    first = false;
  }
}

void completer_main(rg_frontend *f) {
  std::vector<rg_completion> buf(4096);
  while (!f->stop_completer.load()) {
    uint64_t n = 0;
    if (rg_server_poll_wait(f->srv, buf.data(), buf.size(), &n, 2000) != RG_OK) break;
    for (uint64_t i = 0; i < n; i++) {
      if (buf[i].status != RG_OK) f->n_failed++;
      complete(f, buf[i].tag, buf[i].status == RG_OK ? buf[i].version : ~0ull);
    }
  }
}

void wal_main(rg_frontend *f) {
  std::vector<rg_request> ready;
  for (;;) {
    std::unique_lock<std::mutex> lk(f->wmu);
    f->wcv.wait(lk, [&] { return f->wal_stop || f->writing->n > 0; });
    if (f->writing->n == 0) break;  // stopped and empty
    std::swap(f->writing, f->syncing);
    f->writing->version = f->syncing->version + 1;
    f->writing->n = 0;
    lk.unlock();
    f->wcv.notify_all();  // appenders waiting for room
    const off_t at = (off_t)(f->syncing->version - 1) * (off_t)WAL_BLOCK;
    const bool ok = pwrite(f->wal_fd, f->syncing, WAL_BLOCK, at) == (ssize_t)WAL_BLOCK && fdatasync(f->wal_fd) == 0;
    f->n_blocks++;
    lk.lock();
    ready.clear();
    while (!f->pend.empty() && f->pend.front().version <= f->syncing->version) {
      ready.push_back(f->pend.front().req);
      f->pend.pop_front();
    }
    lk.unlock();
    if (!ok) {  // not durable: refuse rather than apply
      for (const rg_request &r : ready) refuse(f, r);
      continue;
    }
    submit(f, ready.data(), ready.size());  // durable: apply in log order
  }
}

}  // namespace

extern "C" {

int rg_frontend_start(rg_server *s, uint32_t instance, const char *host, uint16_t port, const char *wal_path,
                      uint32_t sync_requests, rg_frontend **out) {
  if (!s || !out) {
    rg::set_error("rg_frontend_start: null server or output");
    return RG_EINVAL;
  }
  auto f = std::make_unique<rg_frontend>();
  f->srv = s;
  f->instance = instance;
  f->sync_left = sync_requests;
  f->lfd = socket(AF_INET, SOCK_STREAM, 0);
  if (f->lfd < 0) {
    rg::set_error("rg_frontend_start: socket() failed");
    return RG_EINVAL;
  }
  int one = 1;
  setsockopt(f->lfd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
  sockaddr_in a{};
  a.sin_family = AF_INET;
  a.sin_port = htons(port);
  const char *h = host ? host : "127.0.0.1";
  if (inet_pton(AF_INET, h, &a.sin_addr) != 1 || bind(f->lfd, reinterpret_cast<sockaddr *>(&a), sizeof(a)) != 0 ||
      listen(f->lfd, 128) != 0) {
    close(f->lfd);
    rg::set_error("rg_frontend_start: cannot listen on " + std::string(h) + ":" + std::to_string(port));
    return RG_EINVAL;
  }
  socklen_t len = sizeof(a);
  getsockname(f->lfd, reinterpret_cast<sockaddr *>(&a), &len);
  f->port = ntohs(a.sin_port);
  if (wal_path) {
    f->wal_fd = open(wal_path, O_RDWR | O_CREAT | O_TRUNC, 0644);
    if (f->wal_fd < 0) {
      close(f->lfd);
      rg::set_error(std::string("rg_frontend_start: cannot open the WAL ") + wal_path);
      return RG_EINVAL;
    }
    f->writing = static_cast<WalBlock *>(aligned_alloc(WAL_BLOCK, WAL_BLOCK));
    f->syncing = static_cast<WalBlock *>(aligned_alloc(WAL_BLOCK, WAL_BLOCK));
    std::memset(f->writing, 0, WAL_BLOCK);
    std::memset(f->syncing, 0, WAL_BLOCK);
    f->writing->version = 1;
    f->waler = std::thread(wal_main, f.get());
  }
  f->completer = std::thread(completer_main, f.get());
  f->acceptor = std::thread(acceptor_main, f.get());
  *out = f.release();
  return RG_OK;
}

int rg_frontend_port(rg_frontend *f, uint16_t *port) {
  if (!f || !port) return RG_EINVAL;
  *port = f->port;
  return RG_OK;
}

int rg_frontend_stats_get(rg_frontend *f, rg_frontend_stats *st) {
  if (!f || !st) return RG_EINVAL;
  std::vector<uint64_t> v;
  {
    std::lock_guard<std::mutex> lk(f->smu);
    v = f->lat;
  }
  std::sort(v.begin(), v.end());
  auto pct = [&](double q) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(q * (double)v.size()))] * 1e-3; };
  double sum = 0;
  for (uint64_t x : v) sum += (double)x;
  *st = rg_frontend_stats{f->n_conn.load(), f->n_req.load(), f->n_upd.load(), f->n_sync.load(), f->n_blocks.load(),
                          f->n_failed.load(), f->offset.load(), pct(0.5), pct(0.99), pct(0.999),
                          v.empty() ? 0.0 : v.back() * 1e-3, v.empty() ? 0.0 : sum * 1e-3 / (double)v.size()};
  return RG_OK;
}

int rg_frontend_stop(rg_frontend *f, uint64_t timeout_ms) {
  if (!f) return RG_EINVAL;
  f->stop_accept.store(true);
  if (f->acceptor.joinable()) f->acceptor.join();
  std::vector<std::shared_ptr<Conn>> conns;
  {
    std::lock_guard<std::mutex> lk(f->cmu);
    conns = f->conns;
  }
  for (auto &c : conns) shutdown(c->fd, SHUT_RD);  // no new requests
  for (auto &c : conns)
    if (c->reader.joinable()) c->reader.join();
  // the updates already taken complete (the WAL writer keeps flushing meanwhile)
  int rc = RG_OK;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  while (f->in_flight.load() > 0) {
    if (std::chrono::steady_clock::now() > deadline) {
      rc = RG_ETIMEOUT;
      rg::set_error("rg_frontend_stop: updates still in flight at the timeout");
      break;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
  if (f->wal_fd >= 0) {
    {
      std::lock_guard<std::mutex> lk(f->wmu);
      f->wal_stop = true;
    }
    f->wcv.notify_all();
    if (f->waler.joinable()) f->waler.join();
    fdatasync(f->wal_fd);
    close(f->wal_fd);
    free(f->writing);
    free(f->syncing);
  }
  f->stop_completer.store(true);
  if (f->completer.joinable()) f->completer.join();
  for (auto &c : conns) close(c->fd);
  close(f->lfd);
  delete f;
  return rc;
}

int rg_wal_read(const char *path, rg_wal_record *out, uint64_t cap, uint64_t *n) {
  if (!path || !n || (cap && !out)) return RG_EINVAL;
  int fd = open(path, O_RDONLY);
  if (fd < 0) {
    rg::set_error(std::string("rg_wal_read: cannot open ") + path);
    return RG_EINVAL;
  }
  WalBlock b;
  uint64_t got = 0;
  for (uint64_t k = 0;; k++) {
    if (pread(fd, &b, WAL_BLOCK, (off_t)(k * WAL_BLOCK)) != (ssize_t)WAL_BLOCK) break;
    if (b.version != k + 1 || b.n == 0 || b.n > WAL_RECS) break;
    for (uint64_t i = 0; i < b.n; i++, got++)
      if (got < cap) out[got] = b.rec[i];
  }
  close(fd);
  *n = got;
  return RG_OK;
}

int rg_wal_replay(rg_graph *g, int algo, const char *path, int directed, uint64_t *applied) {
  if (!g) return RG_EINVAL;
  uint64_t n = 0;
  int rc = rg_wal_read(path, nullptr, 0, &n);
  if (rc) return rc;
  std::vector<rg_wal_record> recs(n);
  if ((rc = rg_wal_read(path, recs.data(), n, &n))) return rc;
  std::vector<rg_edge> run;
  for (uint64_t i = 0; i < n;) {
    const uint32_t type = recs[i].type;
    if (type > REQ_DEL) {
      rg::set_error("rg_wal_replay: record of unknown type");
      return RG_EINVAL;
    }
    run.clear();
    for (; i < n && recs[i].type == type; i++) run.push_back(rg_edge{recs[i].src, recs[i].dst, recs[i].data});
    // a run of inserts (or of deletes) commutes, so it applies as one batch
    rc = type == REQ_ADD ? rg_apply_add(g, algo, run.data(), run.size(), directed, nullptr)
                         : rg_apply_del(g, algo, run.data(), run.size(), directed, nullptr);
    if (rc) return rc;
  }
  if (applied) *applied = n;
  return RG_OK;
}

}  // extern "C"
