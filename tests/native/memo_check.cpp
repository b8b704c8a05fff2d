// Host checks of the served form's table of recorded Local_Alignment calls
// (distributedpanga_b200/csrc/memo.h).  Exits non-zero on the first failure.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>

#include "../../distributedpanga_b200/csrc/memo.h"

using namespace pga;

#define CHECK(c)                                               \
  do {                                                         \
    if (!(c)) {                                                \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      std::exit(1);                                            \
    }                                                          \
  } while (0)

int main() {
  std::mt19937_64 rng(7);
  for (int n : {0, 1, 7, 1000, 100000}) {
    // logged calls: keys drawn from a small space (so some repeat), values
    // a function of the first occurrence, every 11th trace not kept
    std::vector<uint32_t> lk(MEMO_KEY * (size_t)n);
    std::vector<int32_t> lv(MEMO_VAL * (size_t)n);
    std::vector<int64_t> lt(n);
    std::map<std::vector<uint32_t>, std::pair<int32_t, int64_t>> first;
    for (int q = 0; q < n; q++) {
      uint32_t *k = &lk[MEMO_KEY * q];
      k[0] = (uint32_t)(rng() % 300) | ((uint32_t)(rng() % 300) << 15) | ((uint32_t)(rng() & 1) << 30);
      for (int i = 1; i < MEMO_KEY; i++) k[i] = (uint32_t)(rng() % 5) - 2u;
      for (int i = 0; i < MEMO_VAL; i++) lv[MEMO_VAL * q + i] = q * 10 + i;
      lt[q] = (q % 11 == 10) ? -1 : (int64_t)q * 3;
      std::vector<uint32_t> kv(k, k + MEMO_KEY);
      if (lt[q] >= 0 && !first.count(kv)) first[kv] = {lv[MEMO_VAL * q], lt[q]};
    }
    const MemoTable T = memo_table(lk.data(), lv.data(), lt.data(), n);
    CHECK((T.cap & (T.cap - 1)) == 0 && T.cap >= 16 && T.cap >= 2 * (int64_t)first.size());
    CHECK(T.entries == (int64_t)first.size());
    for (const auto &kv : first) {
      const int64_t s = memo_find(T, kv.first.data());
      CHECK(s >= 0);
      CHECK(T.val[MEMO_VAL * s] == kv.second.first && T.toff[s] == kv.second.second);
    }
    // a key never logged (contig numbers beyond the drawn range) is absent
    for (int t = 0; t < 200; t++) {
      uint32_t k[MEMO_KEY] = {(uint32_t)(400 + t) | (5u << 15), 1, 2, 3, 4, 5};
      CHECK(memo_find(T, k) < 0);
    }
    std::printf("ok n=%d entries=%lld cap=%lld\n", n, (long long)T.entries, (long long)T.cap);
  }
  return 0;
}
