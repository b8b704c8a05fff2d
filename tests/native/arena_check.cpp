// Host checks of the context arena (distributedpanga_b200/csrc/arena.h)
// against a fake device of fixed capacity.  Prints one line per check and
// exits non-zero on the first failure.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../distributedpanga_b200/csrc/arena.h"

using pga::Arena;

namespace {

const size_t MB = (size_t)1 << 20, GB = (size_t)1 << 30;

// A device of `cap` bytes: addresses from a counter (never reused, never
// dereferenced), 256-byte aligned; tracks what is allocated.
struct FakeDevice {
  size_t cap, used = 0;
  uintptr_t next = 1 << 20;
  std::map<void *, size_t> live;
  int64_t mallocs = 0, frees = 0;
  static int m(void *u, void **p, size_t bytes) {
    FakeDevice *d = (FakeDevice *)u;
    d->mallocs++;
    if (d->used + bytes > d->cap) return 1;
    *p = (void *)d->next;
    d->next += (bytes + 4095) / 4096 * 4096 + 4096;
    d->used += bytes;
    d->live[*p] = bytes;
    return 0;
  }
  static void f(void *u, void *p) {
    FakeDevice *d = (FakeDevice *)u;
    d->frees++;
    auto it = d->live.find(p);
    if (it == d->live.end()) {
      std::printf("FAIL free of an address the device never gave\n");
      std::exit(1);
    }
    d->used -= it->second;
    d->live.erase(it);
  }
};

#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) {                                                    \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);     \
      std::exit(1);                                                \
    }                                                              \
  } while (0)

// Live buffers never overlap and lie inside what the device gave.
struct Live {
  std::map<uintptr_t, size_t> m;
  void add(void *p, size_t n) {
    uintptr_t a = (uintptr_t)p;
    CHECK(a % Arena::ALIGN == 0);
    auto it = m.lower_bound(a);
    if (it != m.end()) CHECK(a + n <= it->first);
    if (it != m.begin()) {
      auto pv = std::prev(it);
      CHECK(pv->first + pv->second <= a);
    }
    m[a] = n;
  }
  void del(void *p) { CHECK(m.erase((uintptr_t)p) == 1); }
};

void basic() {
  FakeDevice d{4 * GB};
  Arena A(FakeDevice::m, FakeDevice::f, &d);
  Live L;
  std::vector<void *> small;
  for (int i = 0; i < 100; i++) {
    size_t n = 1000 + 37 * i;
    void *p = A.alloc(n);
    CHECK(p);
    L.add(p, n);
    small.push_back(p);
  }
  CHECK(A.slabs() == 1 && d.mallocs == 1);  // all in one small slab
  void *big = A.alloc(100 * MB);
  CHECK(big);
  L.add(big, 100 * MB);
  CHECK(A.slabs() == 2);
  // frees coalesce: with every small buffer back, the small slab is one range
  for (void *p : small) {
    CHECK(A.release(p));
    L.del(p);
  }
  CHECK(!A.release((void *)12345));
  CHECK(A.largest_free() == Arena::SMALL_SLAB);
  // best fit: of two free large ranges the smaller one that fits
  void *b2 = A.alloc(300 * MB);
  L.add(b2, 300 * MB);
  CHECK(A.release(big));
  L.del(big);
  CHECK(A.release(b2));
  L.del(b2);
  void *c = A.alloc(90 * MB);
  CHECK(c == big);
  L.add(c, 90 * MB);
  void *e = A.alloc(200 * MB);
  CHECK(e == b2);
  L.add(e, 200 * MB);
  void *f = A.alloc(100 * MB);  // b2's rest (100 MB) fits exactly
  CHECK((uintptr_t)f == (uintptr_t)b2 + 200 * MB);
  L.add(f, 100 * MB);
  const int64_t calls = d.mallocs;
  CHECK(calls == 3);
  A.clear();
  CHECK(d.used == 0 && d.live.empty());
  std::printf("ok basic\n");
}

void trim_when_full() {
  FakeDevice d{GB};
  Arena A(FakeDevice::m, FakeDevice::f, &d);
  void *a = A.alloc(600 * MB);
  CHECK(a);
  CHECK(A.release(a));
  CHECK(A.held_bytes() == 600 * MB && A.free_bytes() == 600 * MB);
  void *b = A.alloc(700 * MB);  // no fit, no room: the empty slab goes back first
  CHECK(b);
  CHECK(A.slabs() == 1 && A.held_bytes() == 700 * MB && d.frees == 1);
  void *c = A.alloc(400 * MB);  // no room even after trimming (b is live)
  CHECK(!c);
  CHECK(A.release(b));
  A.clear();
  CHECK(d.used == 0);
  std::printf("ok trim_when_full\n");
}

// A context's pipeline passes on a 2 x 1 Gbp genome pair (buffer sizes of
// that run), requested the way the context requests them: a range the arena
// holds, else the same after shedding the alignment buffers, else a new slab.
struct Ctx {
  Arena &A;
  std::map<std::string, std::pair<void *, size_t>> buf;
  std::vector<std::string> align_names;
  bool in_align = false;
  int sheds = 0;
  explicit Ctx(Arena &a) : A(a) {}
  bool shed() {
    if (in_align) return false;
    bool any = false;
    for (auto &n : align_names) {
      auto it = buf.find(n);
      if (it != buf.end() && it->second.first) {
        CHECK(A.release(it->second.first));
        it->second = {nullptr, 0};
        any = true;
      }
    }
    sheds += any;
    return any;
  }
  void ensure(const std::string &name, size_t bytes) {
    auto &b = buf[name];
    if (b.second >= bytes) return;
    CHECK(A.release(b.first));
    b = {nullptr, 0};
    void *p = A.fit(bytes);
    if (!p && shed()) p = A.fit(bytes);
    if (!p) p = A.alloc(bytes);
    if (!p) {
      std::printf("FAIL no room for %s (%zu MB): held %zu MB, free %zu MB, largest %zu MB\n", name.c_str(),
                  bytes / MB, A.held_bytes() / MB, A.free_bytes() / MB, A.largest_free() / MB);
      std::exit(1);
    }
    b = {p, bytes};
  }
  void release(const std::string &name) {
    auto &b = buf[name];
    CHECK(A.release(b.first));
    b = {nullptr, 0};
  }
};

void pipeline_passes() {
  FakeDevice d{(size_t)183 * GB};
  Arena A(FakeDevice::m, FakeDevice::f, &d);
  Ctx c(A);
  const size_t nrec = 1586550059ull, nn = 1698799933ull, nc = 640428007ull, seqtot = 1999996444ull;
  c.align_names = {"numf", "numr", "pk", "wave", "points", "cells", "ovl", "perm", "cand", "recs", "outb",
                   "rng_ovl", "tasks", "pout", "pflag", "pidx", "pstart", "pab", "binfo0", "binfo1", "plive0",
                   "plive1", "ftasks", "fout", "lreq"};
  c.ensure("bps", seqtot / 4 + 16);
  c.ensure("dclen", 8 * 7256);
  c.ensure("dboff", 8 * 7256);
  int64_t calls_after[6] = {0};
  for (int pass = 0; pass < 6; pass++) {
    // index build
    c.ensure("hist", 4 * ((1 << 22) + 1));
    c.ensure("start", 4 * ((1 << 24) + 1));
    c.ensure("coarse", 4 * (4 * ((size_t)1 << 22) + 2));
    c.ensure("scan_tmp", 4 * 70000);
    c.ensure("rec", 16 * nrec + 16);
    c.ensure("qmed", 4 << 24);
    c.ensure("qbig", 4 << 24);
    c.ensure("qcount", 32);
    c.ensure("rec2", 16 * (nrec / 12) + 16);
    c.ensure("u64tmp", 8 * 5000);
    c.ensure("lcp", nrec + 16);
    // merge
    c.ensure("blk_n", 4 * (nrec / 256 + 1));
    c.ensure("blk_c", 4 * (nrec / 256 + 1));
    c.ensure("blk_tmp", 4 * (nrec / 256 / 128 + 64));
    c.ensure("seed0", 16 * nn + 16);
    c.ensure("seed1", 16 * nc + 16);
    // diagonal sorts
    c.ensure("keys0", 16 * nn + 16);
    c.ensure("keys_alt", 16 * nn + 16);
    c.ensure("rhist", 4 * (nn / 4096 * 256 + 64));
    c.ensure("rscan", 4 * (nn / 4096 * 256 / 128 + 64));
    c.ensure("keys1", 16 * nc + 16);
    c.ensure("keys_alt", 16 * nc + 16);
    // alignment: what it no longer reads goes first when the device is short
    c.in_align = true;
    const double need = 16.0 * seqtot + 8.0 * (nn + nc) + 8.0 * GB;
    if ((double)(d.cap - d.used) + (double)A.free_bytes() < need)
      for (const char *n : {"rec", "rec2", "lcp", "seed0", "seed1", "keys_alt"}) c.release(n);
    c.ensure("numf", seqtot + 64);
    c.ensure("numr", seqtot + 64);
    c.ensure("pk", seqtot / 4 + 4096);
    c.ensure("binfo0", 8 * nn / 16);
    c.ensure("binfo1", 8 * nc / 16);
    c.ensure("plive0", 101122898);
    c.ensure("plive1", 101122898);
    c.ensure("tasks", 32 * 8129045);
    c.ensure("pout", 48 * 8129045);
    c.ensure("pflag", 101122898);
    c.ensure("pidx", 8 * 101122898);
    c.ensure("pstart", 8 * 101122898);
    c.ensure("pab", 8 * 101122898);
    c.ensure("wave", 592 * 4 * 2 * 65536 * 4);
    c.ensure("points", 592 * 4 * 8 * MB / 4);
    c.ensure("cells", 8 * GB);
    c.ensure("ovl", 592 * 4 * 4096 * 64);
    c.ensure("perm", 592 * 4 * 4096 * 8);
    c.ensure("cand", 4 * GB);
    c.ensure("recs", 64 * 600000);
    c.ensure("outb", 200 * MB);
    c.ensure("rng_ovl", 200 * MB);
    c.ensure("ftasks", 16 * 200000);
    c.ensure("fout", 64 * 200000);
    c.ensure("lreq", 64 * 1302144);
    c.in_align = false;
    calls_after[pass] = A.driver_calls();
  }
  for (int pass = 2; pass < 6; pass++) CHECK(calls_after[pass] == calls_after[1]);
  std::printf("ok pipeline_passes driver_calls_first=%lld later=%lld held_gb=%.1f sheds=%d\n",
              (long long)calls_after[0], (long long)(calls_after[5] - calls_after[0]), A.held_bytes() / (double)GB,
              c.sheds);
  A.clear();
  CHECK(d.used == 0);
}

}  // namespace

int main() {
  basic();
  trim_when_full();
  pipeline_passes();
  return 0;
}
