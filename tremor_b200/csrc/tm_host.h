// Host-side, bit-exact pieces of the scan path (see tm_host.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace tm_host {

constexpr int kZnormBlock = 32;

struct Hit
{
    uint64_t pos;
    float dist;
};

float cc_to_ed(float cc, int m);
float ed_to_cc(float ed, int m);
void znormalize(float *values, int len);
void block_order(const float *q, int m, int *order);
int select_knn(std::vector<Hit> &cands, int k, int merge, std::vector<Hit> &kept);
int extend_knn(const std::vector<Hit> &cands, int k, int merge, std::vector<Hit> &kept);
void threshold_merge(std::vector<Hit> &hits, int merge, std::vector<Hit> &out);

} // namespace tm_host
