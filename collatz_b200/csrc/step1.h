// step1.h -- host Step 1 of the reference's Algorithm 1 (search1,
// collatz_cudav7.cu:497-563): the bit-by-bit tree over the low N-A bits of
// n with the induction (cu:507) and mod-3 path-merging (cu:509-511)
// sieves.  Leaves become pairs (base, T^(N-A)(base) + 1) for Steps 2-3.
#pragma once
#include <stdint.h>

#include <functional>
#include <vector>

namespace cz {

typedef unsigned __int128 u128;

struct Step1Node {
  u128 base;
  uint32_t sigfig, threepower;
  u128 number;
  uint32_t doubleeven, numevens;
};

// Pair layout shared with the cases kernel: base limbs 0..2, bigindex in
// base limb 3 (the reference leaves it 0, cu:201), number limbs 0..3.
inline void pack_pair(uint32_t* w, u128 base, u128 number, uint32_t bigindex) {
  w[0] = (uint32_t)base;
  w[1] = (uint32_t)(base >> 32);
  w[2] = (uint32_t)(base >> 64);
  w[3] = bigindex;
  w[4] = (uint32_t)number;
  w[5] = (uint32_t)(number >> 32);
  w[6] = (uint32_t)(number >> 64);
  w[7] = (uint32_t)(number >> 96);
}

class Step1 {
 public:
  Step1(uint32_t mbi, uint32_t tpo);
  // Subtree roots at sigfig == cut (or leaves reached earlier) in the
  // reference's visiting order.
  void split(const Step1Node& root, uint32_t cut, std::vector<Step1Node>& out) const;
  // All leaves under a node; leaf(bigindex, base, number).
  void leaves(const Step1Node& root, const std::function<void(uint32_t, u128, u128)>& leaf) const;
  // Same, with a plain function pointer for the hot loop.
  typedef void (*LeafFn)(void* ctx, uint32_t bigindex, u128 base, u128 number);
  void leaves_fn(const Step1Node& root, LeafFn fn, void* ctx) const;
  uint32_t mbi() const { return mbi_; }

 private:
  template <class F>
  void rec(u128 base, uint32_t sigfig, uint32_t tp, u128 number, uint32_t de, uint32_t ne, uint32_t cut,
           F& f) const;
  uint32_t mbi_, tpo_;
  u128 p3_[128];
};

}  // namespace cz
