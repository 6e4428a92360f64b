// Host-side CTA split of a batched persistent launch (no CUDA): kept in a header of its
// own so that a plain C++ compiler can test it.
#pragma once
#include <vector>

namespace polar {

// CTA split: one CTA per problem, the rest in proportion to cost (largest remainders),
// each problem capped where its row streams would give a thread fewer than two items.
inline void split_ctas(const std::vector<double>& cost, const std::vector<int>& cap, int total,
                       std::vector<int>& ctas) {
  const int np = (int)cost.size();
  ctas.assign(np, 1);
  int left = total - np;
  double csum = 0.0;
  for (double c : cost) csum += c;
  if (left <= 0 || csum <= 0.0) return;
  std::vector<double> frac(np, 0.0);
  int used = 0;
  for (int b = 0; b < np; ++b) {
    const double want = left * cost[b] / csum;
    int add = (int)want;
    if (ctas[b] + add > cap[b]) add = cap[b] - ctas[b] > 0 ? cap[b] - ctas[b] : 0;
    ctas[b] += add;
    used += add;
    frac[b] = want - (double)(int)want;
  }
  left -= used;
  // hand out the rest one at a time: largest remainder first, then any problem below its cap
  while (left > 0) {
    int best = -1;
    for (int b = 0; b < np; ++b)
      if (ctas[b] < cap[b] && (best < 0 || frac[b] > frac[best])) best = b;
    if (best < 0) break;
    ctas[best] += 1;
    frac[best] = -1.0;
    --left;
    bool any = false;
    for (int b = 0; b < np; ++b) any |= frac[b] >= 0.0 && ctas[b] < cap[b];
    if (!any)
      for (int b = 0; b < np; ++b) frac[b] = cost[b];
  }
}

}  // namespace polar
