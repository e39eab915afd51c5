// step1.cpp -- host Step 1 (search1, collatz_cudav7.cu:497-563).
#include "step1.h"

namespace cz {

static const uint32_t NUMERATOR = 306, DENOMINATOR = 485;

Step1::Step1(uint32_t mbi, uint32_t tpo) : mbi_(mbi), tpo_(tpo) {
  u128 a = 1;
  for (int i = 0; i < 128; i++) {
    p3_[i] = a;  // THREEPOWERS, cu:104-105 (wraps mod 2^128 past 3^80)
    a *= 3;
  }
}

// f(kind, node...) with kind 0 = leaf (sigfig == N-A), 1 = cut root.
template <class F>
void Step1::rec(u128 base, uint32_t sigfig, uint32_t tp, u128 number, uint32_t de, uint32_t ne, uint32_t cut,
                F& f) const {
  // Induction sieve (cu:507); u32 arithmetic as in the reference.
  if (DENOMINATOR * tp <= NUMERATOR * sigfig) return;
  // Mod 3 preimage sieve (cu:509-511).
  if (ne >= 2 && ne % 2 == 0) {
    if (NUMERATOR * (sigfig - 1) >= DENOMINATOR * (tp - 1)) return;
  }
  if (sigfig == mbi_) {
    f(0, base, sigfig, tp, number, de, ne);
    return;
  }
  if (sigfig == cut) {
    f(1, base, sigfig, tp, number, de, ne);
    return;
  }
  const uint32_t doubleinplay = (NUMERATOR * (sigfig + 1) >= DENOMINATOR * tp) ? 1u : 0u;  // cu:543
  const u128 numberA = number;
  const u128 numberB = number + p3_[tp & 127];
  if (number % 2 == 0) {  // cu:548-554
    rec(base, sigfig + 1, tp + 1, numberA + numberA / 2, (de | doubleinplay) & ~2u, 0, cut, f);
    if (de < 2) rec(base | ((u128)1 << sigfig), sigfig + 1, tp, numberB / 2 + 1, de << 1, ne + 1, cut, f);
  } else {  // cu:555-561
    if (de < 2) rec(base, sigfig + 1, tp, numberA / 2 + 1, de << 1, ne + 1, cut, f);
    rec(base | ((u128)1 << sigfig), sigfig + 1, tp + 1, numberB + numberB / 2, (de | doubleinplay) & ~2u, 0, cut,
        f);
  }
}

void Step1::split(const Step1Node& r, uint32_t cut, std::vector<Step1Node>& out) const {
  auto f = [&](int, u128 b, uint32_t sf, uint32_t tp, u128 num, uint32_t de, uint32_t ne) {
    out.push_back(Step1Node{b, sf, tp, num, de, ne});
  };
  rec(r.base, r.sigfig, r.threepower, r.number, r.doubleeven, r.numevens, cut, f);
}

void Step1::leaves(const Step1Node& r, const std::function<void(uint32_t, u128, u128)>& leaf) const {
  auto f = [&](int, u128 b, uint32_t, uint32_t tp, u128 num, uint32_t, uint32_t) { leaf(tp - tpo_, b, num); };
  rec(r.base, r.sigfig, r.threepower, r.number, r.doubleeven, r.numevens, 0xFFFFFFFFu, f);
}

void Step1::leaves_fn(const Step1Node& r, LeafFn fn, void* ctx) const {
  auto f = [&](int, u128 b, uint32_t, uint32_t tp, u128 num, uint32_t, uint32_t) { fn(ctx, tp - tpo_, b, num); };
  rec(r.base, r.sigfig, r.threepower, r.number, r.doubleeven, r.numevens, 0xFFFFFFFFu, f);
}

}  // namespace cz
