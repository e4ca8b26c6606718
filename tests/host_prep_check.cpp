// CPU check of the engine's host-side layout preparation (csrc/host_prep.hpp), built by
// tests/test_host_prep.py with AddressSanitizer and UBSan. Prints "ALL OK" or the first failure.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>

#include "host_prep.hpp"

using namespace fb;

#define CHECK(c)                                                                   \
    do {                                                                           \
        if (!(c)) {                                                                \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);               \
            std::exit(1);                                                          \
        }                                                                          \
    } while (0)

struct Csr {
    std::vector<int64_t> ip;
    std::vector<int32_t> ix;
    std::vector<float> d;
};

static Csr random_csr(std::mt19937_64& g, int64_t n, int max_deg, bool integral)
{
    Csr c;
    c.ip.push_back(0);
    std::uniform_int_distribution<int> deg(0, max_deg);
    for (int64_t i = 0; i < n; i++) {
        std::set<int32_t> cols;
        const int k = std::min<int64_t>(deg(g), n);
        while ((int)cols.size() < k) cols.insert((int32_t)(g() % n));
        std::vector<int32_t> v(cols.begin(), cols.end());
        std::shuffle(v.begin(), v.end(), g);   // unsorted columns within the row
        for (int32_t x : v) {
            c.ix.push_back(x);
            const double w = integral ? (double)((int)(g() % 41) - 20) : ((int)(g() % 2001) - 1000) / 37.0;
            c.d.push_back((float)(w == 0 ? 1 : w));
        }
        c.ip.push_back((int64_t)c.ix.size());
    }
    return c;
}

int main()
{
    std::mt19937_64 g(1234);
    const float wsyn = 0.275f;
    for (int trial = 0; trial < 60; trial++) {
        const int64_t n = 1 + (int64_t)(g() % 700);
        const bool integral = trial % 2 == 0;
        const int max_deg = trial % 5 == 0 ? 600 : 40;
        Csr c = random_csr(g, n, max_deg, integral);
        const int64_t nnz = (int64_t)c.ix.size();
        HostCsr H;
        std::string e = prepare_csr(c.ip.data(), c.ix.data(), c.d.data(), n, nnz, wsyn, false, H);
        CHECK(e.empty());
        CHECK(H.acc_mode == (integral ? 0 : 1));
        CHECK((int64_t)H.rp.size() == n + 1 && H.rp[0] == 0);
        int64_t chunks = 0;
        for (int64_t i = 0; i < n; i++) {
            const int64_t len = c.ip[i + 1] - c.ip[i];
            const int64_t pad = H.rp[i + 1] - H.rp[i];
            CHECK(pad % 8 == 0 && pad >= len && pad < len + 8);
            chunks += (pad + 255) / 256;
            std::vector<int32_t> want(c.ix.begin() + c.ip[i], c.ix.begin() + c.ip[i + 1]);
            std::sort(want.begin(), want.end());
            for (int64_t k = 0; k < len; k++) {
                CHECK(H.ix[c.ip[i] + k] == want[k]);
                CHECK(H.pcol[H.rp[i] + k] == want[k]);
                // the weight travelled with its column
                int64_t src = -1;
                for (int64_t q = c.ip[i]; q < c.ip[i + 1]; q++)
                    if (c.ix[q] == want[k]) src = q;
                CHECK(H.wd[c.ip[i] + k] == c.d[src] * wsyn);
                if (integral) CHECK(H.pcnt[H.rp[i] + k] == (int16_t)c.d[src]);
                else CHECK(H.pwfx[H.rp[i] + k] == q32_host(c.d[src] * wsyn));
            }
            for (int64_t k = len; k < pad; k++) {
                CHECK(H.pcol[H.rp[i] + k] == 0);
                if (integral) CHECK(H.pcnt[H.rp[i] + k] == 0);
                else CHECK(H.pwfx[H.rp[i] + k] == 0);
            }
        }
        CHECK(chunks == H.chunks_all);
        // segment capacity: brute force over the pairs of a group of 1..3 instances
        {
            const int64_t n_pad = (n + 15) / 16 * 16;
            const int64_t group = 1 + trial % 3, pairs = group * n_pad;
            const int64_t n_seg = 1 + (int64_t)(g() % 9);
            const int64_t seg_pairs = ((pairs + n_seg - 1) / n_seg + 15) / 16 * 16;
            int64_t want = 1;
            for (int64_t s = 0; s < n_seg; s++) {
                int64_t items = 0;
                for (int64_t p = s * seg_pairs; p < std::min((s + 1) * seg_pairs, pairs); p++) {
                    const int64_t i = p % n_pad;
                    if (i < n) items += (H.rp[i + 1] - H.rp[i] + 255) / 256;
                }
                want = std::max(want, items);
            }
            CHECK(segment_capacity(H, n_pad, group, seg_pairs, n_seg) == want);
        }

        // the by-postsynaptic copy holds every entry once, in pre order within each column
        {
            HostCsc Cc;
            build_csc(H, Cc);
            CHECK((int64_t)Cc.colptr.size() == n + 1 && Cc.colptr[n] == nnz);
            std::vector<int64_t> seen(n, 0);
            for (int64_t j = 0; j < n; j++)
                for (int64_t q = Cc.colptr[j]; q < Cc.colptr[j + 1]; q++) {
                    const int32_t i = Cc.pre[q];
                    if (q > Cc.colptr[j]) CHECK(Cc.pre[q - 1] < i);
                    int64_t k = H.ip[i];
                    while (k < H.ip[i + 1] && H.ix[k] != j) k++;
                    CHECK(k < H.ip[i + 1]);
                    const int64_t src = H.rp[i] + (k - H.ip[i]);
                    if (integral) CHECK(Cc.cnt[q] == H.pcnt[src]);
                    else CHECK(Cc.wfx[q] == H.pwfx[src]);
                    seen[j]++;
                }
        }
        // plastic plans: a random subset, then a superset; weights and ring survive the re-plan
        if (nnz == 0) continue;
        std::vector<int64_t> pos1, pos2;
        for (int64_t k = 0; k < nnz; k++) {
            if (g() % 5 == 0) pos1.push_back(k);
            if (g() % 3 == 0) pos2.push_back(k);
        }
        pos2.insert(pos2.end(), pos1.begin(), pos1.end());
        PlasticPlan P1, P2;
        CHECK(plan_plastic(H, pos1, P1).empty());
        CHECK(plan_plastic(H, pos2, P2).empty());
        for (const PlasticPlan* P : {&P1, &P2}) {
            CHECK((int64_t)P->plr.size() == n + 1 && P->plr[n] == P->n_pl);
            for (int64_t k = 0; k < P->n_pl; k++) {
                const int64_t p = P->pos[k];
                int64_t row = 0;
                while (c.ip[row + 1] <= p) row++;
                CHECK(P->plr[row] <= k && k < P->plr[row + 1]);
                CHECK(P->pre[k] == row && P->post[k] == H.ix[p]);
                CHECK(P->ppost_of[H.ix[p]] == P->pl_pidx[k]);
                CHECK(P->ppost_neuron[P->pl_pidx[k]] == H.ix[p]);
                CHECK(P->w0[k] == H.wd[p] && P->q0[k] == q32_host(H.wd[p]));
            }
        }
        const int32_t B = 3;
        std::vector<float> pw1((size_t)B * P1.n_pl);
        for (size_t k = 0; k < pw1.size(); k++) pw1[k] = (float)k * 0.5f;
        std::vector<float> pw2 = remap_weights(P1, pw1, P2, B);
        for (int64_t k = 0; k < P1.n_pl; k++) {
            const int64_t j = std::lower_bound(P2.pos.begin(), P2.pos.end(), P1.pos[k]) - P2.pos.begin();
            for (int32_t b = 0; b < B; b++) CHECK(pw2[(size_t)b * P2.n_pl + j] == pw1[(size_t)b * P1.n_pl + k]);
        }
        const int64_t rows = 4 * B;
        std::vector<int64_t> ring1((size_t)rows * std::max(1, P1.n_ppost));
        for (size_t k = 0; k < ring1.size(); k++) ring1[k] = (int64_t)k + 1;
        std::vector<int64_t> ring2 = remap_ring(P1, ring1, P2, rows);
        for (int64_t r = 0; r < rows; r++)
            for (int64_t i = 0; i < n; i++)
                if (P1.ppost_of[i] >= 0)
                    CHECK(ring2[(size_t)r * P2.n_ppost + P2.ppost_of[i]] == ring1[(size_t)r * P1.n_ppost + P1.ppost_of[i]]);
    }
    // rejected inputs
    {
        int64_t ip[3] = {0, 2, 3};
        int32_t ix[3] = {1, 1, 0};
        float d[3] = {1, 2, 3};
        HostCsr H;
        CHECK(prepare_csr(ip, ix, d, 2, 3, wsyn, false, H).find("duplicate") != std::string::npos);
        ix[1] = 7;
        CHECK(prepare_csr(ip, ix, d, 2, 3, wsyn, false, H).find("out of range") != std::string::npos);
        int64_t bad[3] = {0, 3, 2};
        ix[1] = 0;
        CHECK(!prepare_csr(bad, ix, d, 2, 2, wsyn, false, H).empty());
        PlasticPlan P;
        int32_t ok_ix[3] = {0, 1, 0};
        CHECK(prepare_csr(ip, ok_ix, d, 2, 3, wsyn, false, H).empty());
        CHECK(!plan_plastic(H, {5}, P).empty());
        CHECK(prepare_csr(ip, ok_ix, d, 2, 3, wsyn, true, H).empty() && H.acc_mode == 1);
    }
    std::printf("ALL OK\n");
    return 0;
}
