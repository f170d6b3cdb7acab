// ibp_oracle_shuffle.cpp -- the reference's k-means seeding, for the oracle.
//
// TEST INFRASTRUCTURE ONLY.  include/preproc/ibp_preproc_host.cuh:176-188 fills a
// std::vector<int> with 0..n-1, calls std::random_shuffle (libstdc++, driven by the
// process rand() state, never srand'd there) and seeds centroid i with row indices[i].
// This file calls the same library routine so the oracle can reproduce that seeding.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "ibp_oracle.h"

extern "C" void orc_random_shuffle_init(int64_t n, int c, int64_t *init, int reseed) {
    if (reseed) std::srand(1);
    std::vector<int> indices((size_t)n);
    for (int64_t i = 0; i < n; ++i) indices[(size_t)i] = (int)i;
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wdeprecated-declarations"
    std::random_shuffle(indices.begin(), indices.end());
#pragma GCC diagnostic pop
    int64_t seeded = (int64_t)c < n ? (int64_t)c : n;
    for (int64_t i = 0; i < seeded; ++i) init[i] = indices[(size_t)i];
}
