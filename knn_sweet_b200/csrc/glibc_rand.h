// glibc_rand.h -- a reentrant restatement of glibc's srand()/rand().
//
// The reference draws its representative rows with the C library generator
// after srand(2015) (src/knnjoin.cu:199-202, 226-229).  glibc's default
// rand() is the TYPE_3 additive feedback generator, whose published
// description is:
//   r[0] = seed (0 is treated as 1)
//   r[i] = 16807 * r[i-1] mod (2^31 - 1)        for i = 1 .. 30
//   r[i] = r[i-31]                               for i = 31 .. 33
//   r[i] = r[i-31] + r[i-3]  (mod 2^32)          for i >= 34
//   the first 310 values past r[33] are discarded; output k is r[k+344] >> 1.
// Keeping the state in an object (instead of the C library's global state)
// lets concurrent calls draw independently; the tests check the sequence
// against the C library's rand().
#pragma once

#include <stdint.h>

namespace knnsweet {

class GlibcRand {
 public:
  explicit GlibcRand(uint32_t seed) {
    int64_t r[344];
    if (seed == 0) seed = 1;
    r[0] = (int32_t)seed;
    for (int i = 1; i < 31; i++) {
      int64_t v = (16807LL * r[i - 1]) % 2147483647LL;
      if (v < 0) v += 2147483647LL;
      r[i] = v;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (int i = 34; i < 344; i++)
      r[i] = (int64_t)(uint32_t)((uint32_t)r[i - 31] + (uint32_t)r[i - 3]);
    for (int i = 0; i < 34; i++) ring_[i] = (uint32_t)r[310 + i];
    pos_ = 0;
  }

  // Next value in [0, 2^31).
  int32_t next() {
    uint32_t v = ring_[(pos_ + 3) % 34] + ring_[(pos_ + 31) % 34];
    ring_[pos_] = v;
    pos_ = (pos_ + 1) % 34;
    return (int32_t)(v >> 1);
  }

 private:
  uint32_t ring_[34];  // r[i-34 .. i-1], oldest at pos_
  int pos_;
};

}  // namespace knnsweet
