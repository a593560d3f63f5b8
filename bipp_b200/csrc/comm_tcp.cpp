// Sum-to-root reduction of float arrays over TCP: the transport of the C++ API's
// Communicator::world() (the reference reduces its images with MPI_Reduce,
// src/image_synthesis.cpp:140-147). Rank 0 listens, the other ranks connect (with
// retries), send (rank, count, data) and wait for rank 0's acknowledgement; rank 0 adds
// the arrays in rank order, so that the sum does not depend on arrival order. Every wait
// is bounded (BIPP_B200_REDUCE_TIMEOUT seconds, default 300).
#include <arpa/inet.h>
#include <netdb.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <poll.h>
#include <sys/socket.h>
#include <unistd.h>

#include <cerrno>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace bippb200 {
namespace {

using Clock = std::chrono::steady_clock;

struct Fd {
  int fd = -1;
  explicit Fd(int f = -1) : fd(f) {}
  Fd(const Fd&) = delete;
  Fd& operator=(const Fd&) = delete;
  Fd(Fd&& o) noexcept : fd(o.fd) { o.fd = -1; }
  Fd& operator=(Fd&& o) noexcept {
    if (this != &o) {
      if (fd >= 0) close(fd);
      fd = o.fd;
      o.fd = -1;
    }
    return *this;
  }
  ~Fd() {
    if (fd >= 0) close(fd);
  }
};

[[noreturn]] void fail(const std::string& what) { throw std::runtime_error("image reduction over TCP: " + what); }

double remaining(Clock::time_point end) {
  return std::chrono::duration<double>(end - Clock::now()).count();
}

void wait_fd(int fd, short ev, Clock::time_point end) {
  for (;;) {
    const double left = remaining(end);
    if (left <= 0) fail("timed out");
    pollfd p{fd, ev, 0};
    const int r = poll(&p, 1, (int)std::min(1000.0, left * 1000.0) + 1);
    if (r > 0) return;
    if (r < 0 && errno != EINTR) fail(std::string("poll: ") + std::strerror(errno));
  }
}

void send_all(int fd, const void* buf, size_t n, Clock::time_point end) {
  const char* p = static_cast<const char*>(buf);
  while (n) {
    wait_fd(fd, POLLOUT, end);
    const ssize_t k = send(fd, p, n, MSG_NOSIGNAL);
    if (k < 0) {
      if (errno == EINTR || errno == EAGAIN) continue;
      fail(std::string("send: ") + std::strerror(errno));
    }
    p += k;
    n -= (size_t)k;
  }
}

void recv_all(int fd, void* buf, size_t n, Clock::time_point end) {
  char* p = static_cast<char*>(buf);
  while (n) {
    wait_fd(fd, POLLIN, end);
    const ssize_t k = recv(fd, p, n, 0);
    if (k == 0) fail("peer closed the connection");
    if (k < 0) {
      if (errno == EINTR || errno == EAGAIN) continue;
      fail(std::string("recv: ") + std::strerror(errno));
    }
    p += k;
    n -= (size_t)k;
  }
}

sockaddr_in resolve(const char* host, int port) {
  addrinfo hints{};
  hints.ai_family = AF_INET;
  hints.ai_socktype = SOCK_STREAM;
  addrinfo* res = nullptr;
  if (getaddrinfo(host, nullptr, &hints, &res) != 0 || !res) fail(std::string("cannot resolve ") + host);
  sockaddr_in a = *reinterpret_cast<sockaddr_in*>(res->ai_addr);
  freeaddrinfo(res);
  a.sin_port = htons((uint16_t)port);
  return a;
}

}  // namespace

void tcp_reduce_sum_to_root(const char* host, int port, size_t rank, size_t size, float* data, size_t count,
                            double timeoutSec) {
  if (size <= 1) return;
  const auto end = Clock::now() + std::chrono::milliseconds((long long)(timeoutSec * 1000));
  const sockaddr_in addr = resolve(host, port);
  const uint64_t magic = 0x62697070b200ull;
  if (rank == 0) {
    Fd ls(socket(AF_INET, SOCK_STREAM, 0));
    if (ls.fd < 0) fail("socket");
    int one = 1;
    setsockopt(ls.fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
    if (bind(ls.fd, reinterpret_cast<const sockaddr*>(&addr), sizeof(addr)) != 0)
      fail("bind to port " + std::to_string(port) + ": " + std::strerror(errno));
    if (listen(ls.fd, (int)size) != 0) fail("listen");
    std::vector<std::vector<float>> parts(size);
    std::vector<Fd> peers;
    for (size_t got = 1; got < size; ++got) {
      wait_fd(ls.fd, POLLIN, end);
      Fd c(accept(ls.fd, nullptr, nullptr));
      if (c.fd < 0) fail("accept");
      uint64_t hdr[3];
      recv_all(c.fd, hdr, sizeof(hdr), end);
      if (hdr[0] != magic || hdr[1] == 0 || hdr[1] >= size || hdr[2] != count) fail("mismatched peer message");
      if (!parts[hdr[1]].empty()) fail("rank " + std::to_string(hdr[1]) + " connected twice");
      parts[hdr[1]].resize(count);
      recv_all(c.fd, parts[hdr[1]].data(), count * sizeof(float), end);
      peers.push_back(std::move(c));
    }
    for (size_t r = 1; r < size; ++r)
      for (size_t i = 0; i < count; ++i) data[i] += parts[r][i];
    const char ack = 1;
    for (auto& p : peers) send_all(p.fd, &ack, 1, end);
  } else {
    Fd c(-1);
    for (;;) {
      c = Fd(socket(AF_INET, SOCK_STREAM, 0));
      if (c.fd < 0) fail("socket");
      if (connect(c.fd, reinterpret_cast<const sockaddr*>(&addr), sizeof(addr)) == 0) break;
      if (remaining(end) <= 0) fail("could not connect to rank 0 on port " + std::to_string(port));
      std::this_thread::sleep_for(std::chrono::milliseconds(50));
    }
    const uint64_t hdr[3] = {magic, (uint64_t)rank, (uint64_t)count};
    send_all(c.fd, hdr, sizeof(hdr), end);
    send_all(c.fd, data, count * sizeof(float), end);
    char ack = 0;
    recv_all(c.fd, &ack, 1, end);
  }
}

}  // namespace bippb200
