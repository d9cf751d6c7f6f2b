// The surface-area plan of the 8-wide collapse (Wide8PlanNode, Wide8Gather in
// bulbit_b200/csrc/wide8_build.cuh), on the host, against brute force: over
// SAH trees of 1 to 40 random boxes (bbg_bvh_build, the reference's build),
// the plan's cost equals the least summed surface area of wide nodes over
// every valid collapse (each wide node holds at most eight children, each a
// binary leaf or a binary node that is a wide node of its own), the collapse
// it gathers has that cost, every leaf is reached exactly once and no wide
// node holds more than eight children. Prints one line per failure and
// returns non-zero if any.
#include "bbg.h"
#include "wide8_build.cuh"

#include <cmath>
#include <cstdio>
#include <random>
#include <set>
#include <vector>

using namespace bbg;

namespace
{

double Area(const bbg_bvh_node& x)
{
    Child8 c;
    for (int a = 0; a < 3; ++a)
    {
        c.lo[a] = x.bmin[a];
        c.hi[a] = x.bmax[a];
    }
    return Wide8Area(c);
}

// Every frontier of the subtree of y (y itself, or a frontier of each child)
// with at most eight members.
void Frontiers(const std::vector<bbg_bvh_node>& nd, int32_t y, std::vector<std::vector<int32_t>>* out)
{
    out->push_back({ y });
    if (nd[y].count > 0)
    {
        return;
    }
    std::vector<std::vector<int32_t>> l, r;
    Frontiers(nd, y + 1, &l);
    Frontiers(nd, nd[y].offset, &r);
    for (const auto& a : l)
    {
        for (const auto& b : r)
        {
            if (a.size() + b.size() <= 8)
            {
                std::vector<int32_t> f(a);
                f.insert(f.end(), b.begin(), b.end());
                out->push_back(f);
            }
        }
    }
}

// Least cost of interior node x as a wide node: its area plus the best
// frontier below it (x excluded) whose interior members are wide nodes.
double Best(const std::vector<bbg_bvh_node>& nd, int32_t x, std::vector<double>* memo)
{
    if ((*memo)[x] >= 0)
    {
        return (*memo)[x];
    }
    std::vector<std::vector<int32_t>> l, r;
    Frontiers(nd, x + 1, &l);
    Frontiers(nd, nd[x].offset, &r);
    double best = 1e300;
    for (const auto& a : l)
    {
        for (const auto& b : r)
        {
            if (a.size() + b.size() > 8)
            {
                continue;
            }
            double v = 0;
            for (const auto* f : { &a, &b })
            {
                for (int32_t c : *f)
                {
                    if (nd[c].count == 0)
                    {
                        v += Best(nd, c, memo);
                    }
                }
            }
            best = std::min(best, v);
        }
    }
    (*memo)[x] = Area(nd[x]) + best;
    return (*memo)[x];
}

} // namespace

int main()
{
    int failures = 0, trees = 0;
    for (int n = 1; n <= 40; ++n)
    {
        for (int seed = 0; seed < 6; ++seed)
        {
            std::mt19937 rng(uint32_t(1000 * n + seed));
            std::uniform_real_distribution<float> u(-1.0f, 1.0f), h(0.01f, 0.4f);
            std::vector<float> boxes(6 * size_t(n));
            for (int i = 0; i < n; ++i)
            {
                for (int a = 0; a < 3; ++a)
                {
                    const float c = u(rng), e = (seed % 2) ? h(rng) : 0.05f; // uniform or mixed sizes
                    boxes[6 * i + a] = c - e;
                    boxes[6 * i + 3 + a] = c + e;
                }
            }
            std::vector<bbg_bvh_node> nd(2 * size_t(n));
            std::vector<int32_t> slots(n);
            int32_t nn = 0;
            if (bbg_bvh_build(boxes.data(), n, nd.data(), slots.data(), &nn) != BBG_OK)
            {
                std::printf("n=%d seed=%d: bbg_bvh_build failed\n", n, seed);
                ++failures;
                continue;
            }
            nd.resize(nn);
            ++trees;
            std::vector<float> cost(8 * nd.size(), 0.0f);
            std::vector<uint8_t> split(8 * nd.size(), 0);
            for (size_t b = nd.size(); b-- > 0;)
            {
                if (nd[b].count == 0)
                {
                    Wide8PlanNode(nd[b], &cost[8 * (b + 1)], &cost[8 * size_t(nd[b].offset)], &cost[8 * b], &split[8 * b]);
                }
            }
            // The collapse the plan gathers: wide nodes breadth first.
            std::vector<int32_t> queue{ 0 };
            std::multiset<int32_t> leaves;
            double realised = 0;
            bool bad = false;
            for (size_t q = 0; q < queue.size(); ++q)
            {
                int32_t kids[8];
                const int k = Wide8Gather(nd.data(), split.data(), queue[q], kids);
                bad |= k < 1 || k > 8;
                if (nd[queue[q]].count == 0)
                {
                    realised += Area(nd[queue[q]]);
                }
                for (int c = 0; c < k; ++c)
                {
                    if (nd[kids[c]].count > 0)
                    {
                        leaves.insert(kids[c]);
                    }
                    else
                    {
                        queue.push_back(kids[c]);
                    }
                }
            }
            int n_leaves = 0;
            for (int32_t b = 0; b < nn; ++b)
            {
                if (nd[b].count > 0)
                {
                    ++n_leaves;
                    bad |= leaves.count(b) != 1;
                }
            }
            bad |= int(leaves.size()) != n_leaves;
            if (nd[0].count == 0)
            {
                std::vector<double> memo(nd.size(), -1.0);
                const double brute = Best(nd, 0, &memo);
                const double planned = cost[0];
                const double tol = 1e-5 * brute;
                if (std::fabs(planned - brute) > tol || std::fabs(realised - brute) > tol)
                {
                    std::printf("n=%d seed=%d: plan %.9g, gathered %.9g, brute force %.9g\n", n, seed, planned,
                                realised, brute);
                    ++failures;
                }
            }
            if (bad)
            {
                std::printf("n=%d seed=%d: leaves or child counts wrong\n", n, seed);
                ++failures;
            }
        }
    }
    std::printf("%d trees, %d failures\n", trees, failures);
    return failures ? 1 : 0;
}
