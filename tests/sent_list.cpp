// A randomized check of the TCP sent list (twins_b200/csrc/tb_tcp.cuh: SentList, its flag words
// of eight positions and the word-wise shifts of open / join_previous), built with g++ for the host
// by tests/test_sent_list.py. Random opens, joins, flag changes and whole-list losses on rings of
// every capacity class, with the head anywhere (so that shifts wrap), and ACKs that drop and cut
// items are mirrored on a plain per-item model; after every step each item's flags, the byte counters (lost, retransmitted,
// sacked, candidates), the sacked-item count and the candidate search bound must agree with it.
// Exit status 0: all agree.
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

struct uint4 // (the frame copies of the included headers name CUDA's vector type; unused here)
{
    unsigned x, y, z, w;
};
#include "tb_tcp.cuh"

using namespace tb;

namespace
{
struct Item
{
    uint32_t start;
    uint8_t f;
};

bool check(const SentList &L, const SndRec &S, const std::vector<Item> &m, uint32_t high, int trial, int op)
{
    uint32_t lost = 0, retx = 0, sack = 0, cand = 0, sack_n = 0, first_cand = (uint32_t)m.size();
    for (size_t j = 0; j < m.size(); j++)
    {
        const uint32_t len = (j + 1 < m.size() ? m[j + 1].start : high) - m[j].start;
        if (L.flags((uint32_t)j) != m[j].f || L.beg((uint32_t)j) != m[j].start)
        {
            printf("trial %d op %d: item %zu flags %u start %u, model %u %u\n", trial, op, j, L.flags((uint32_t)j), L.beg((uint32_t)j), m[j].f,
                   m[j].start);
            return false;
        }
        lost += (m[j].f & FL_LOST) ? len : 0;
        retx += (m[j].f & FL_RETX) ? len : 0;
        sack += (m[j].f & FL_SACK) ? len : 0;
        sack_n += (m[j].f & FL_SACK) ? 1 : 0;
        if (SentList::candidate(m[j].f))
        {
            cand += len;
            if (first_cand == m.size())
                first_cand = (uint32_t)j;
        }
    }
    if (S.it_n != m.size() || S.lost_b != lost || S.rtx_b != retx || S.sack_b != sack || S.cand_b != cand || S.sack_n != sack_n ||
        (first_cand < m.size() && S.cand_lo > first_cand))
    {
        printf("trial %d op %d: counters n %u lost %u/%u retx %u/%u sack %u/%u cand %u/%u sacked %u/%u bound %u first %u\n", trial, op, S.it_n,
               S.lost_b, lost, S.rtx_b, retx, S.sack_b, sack, S.cand_b, cand, S.sack_n, sack_n, S.cand_lo, first_cand);
        return false;
    }
    return true;
}
} // namespace

int main()
{
    std::mt19937 g(7);
    for (int trial = 0; trial < 4000; trial++)
    {
        const uint32_t cap = 8 * (1 + g() % 6);
        std::vector<uint32_t> st(cap);
        std::vector<uint8_t> fl(cap / 2 + 8);
        for (auto &b : fl)
            b = (uint8_t)g(); // (stale bits: never read)
        Sim s{};
        s.it_start = st.data();
        s.it_fl = fl.data();
        SndRec S{};
        S.it_cap = cap;
        S.it_head = g() % cap;
        S.una = 0;
        std::vector<Item> m;
        uint32_t high = 0;
        S.high = high;
        SentList L(s, S);
        unsigned ovf = 0;
        for (int op = 0; op < 300; op++)
        {
            const int k = (int)(g() % 10);
            if (k < 2 && S.it_n < cap)
            {
                // new data: an item at the end, clean, from `high` on
                const uint32_t seq = high;
                high += 1 + g() % 3000;
                S.high = high;
                L.open(S.it_n, seq, 0, ovf);
                m.push_back(Item{seq, 0});
            }
            else if (k < 4 && S.it_n && S.it_n < cap)
            {
                // a split: item i - 1 keeps its first bytes, the rest becomes item i with its flags
                const uint32_t i = 1 + g() % S.it_n;
                const uint32_t lo = m[i - 1].start, hi = i < m.size() ? m[i].start : high;
                if (hi - lo < 2)
                    continue;
                const uint32_t seq = lo + 1 + g() % (hi - lo - 1);
                L.open(i, seq, m[i - 1].f, ovf);
                m.insert(m.begin() + i, Item{seq, m[i - 1].f});
            }
            else if (k < 6 && S.it_n >= 2)
            {
                // item i joins item i - 1 once they agree on everything (as a retransmission joins)
                const uint32_t i = 1 + g() % (S.it_n - 1);
                if (m[i].f != m[i - 1].f)
                {
                    L.mark(i, m[i - 1].f);
                    m[i].f = m[i - 1].f;
                }
                L.join_previous(i);
                m.erase(m.begin() + i);
            }
            else if (k < 9 && S.it_n)
            {
                const uint32_t i = g() % S.it_n;
                const uint8_t f = (uint8_t)(g() % 8);
                L.mark(i, f);
                m[i].f = f;
            }
            else if (k == 9 && S.it_n && (g() & 1))
            {
                // an ACK: the items below it leave, an item it falls inside is cut there (an ACK
                // leaving a sacked item first is left out: the Reno emulation's follow-up is not modelled)
                const uint32_t ack = m[0].start + g() % (high - m[0].start + 1);
                size_t j = 0;
                while (j < m.size() && (j + 1 < m.size() ? m[j + 1].start : high) <= ack)
                    j++;
                if (j < m.size() && (m[j].f & FL_SACK))
                    continue;
                const uint32_t gone = j < m.size() ? (m[j].start < ack ? m[j].start : ack) - m[0].start : high - m[0].start;
                m.erase(m.begin(), m.begin() + j);
                if (!m.empty() && m[0].start < ack)
                    m[0].start = ack;
                if (ack_drop(L, ack) != gone)
                {
                    printf("trial %d op %d: ack %u returned bytes differ from %u\n", trial, op, ack, gone);
                    return 1;
                }
            }
            else if (S.it_n)
            {
                S.una = m[0].start;
                everything_lost(L);
                for (auto &x : m)
                    x.f = FL_LOST;
            }
            if (!check(L, S, m, high, trial, op))
                return 1;
        }
    }
    puts("sent list: all agree");
    // the RTT history: first sends, retransmissions (some reaching past the next entry), ACKs,
    // against a list scanned from the oldest entry every time
    for (int trial = 0; trial < 3000; trial++)
    {
        const uint32_t cap = 8 * (1 + g() % 6);
        std::vector<uint32_t> lo(cap), hi(cap);
        std::vector<int64_t> at(cap);
        Sim s{};
        s.h_seq = lo.data();
        s.h_end = hi.data();
        s.h_t = at.data();
        SndRec S{};
        S.it_cap = cap;
        S.h_head = g() % cap;
        S.srtt = 0;
        struct E
        {
            uint32_t lo, hi;
            int64_t at;
        };
        std::vector<E> m;
        uint32_t high = 1000, una = 1000;
        unsigned ovf = 0;
        for (int op = 0; op < 200; op++)
        {
            RttLog log(s, S);
            const int k = (int)(g() % 10);
            if (k < 4)
            {
                const uint32_t len = 1 + g() % 1500;
                log.first_send(high, len, op, ovf);
                if (m.size() < cap)
                    m.push_back(E{high, high + len, op});
                high += len;
            }
            else if (k < 8 && high > una)
            {
                const uint32_t seq = una + g() % (high - una), len = 1 + g() % (g() % 4 ? 1500 : 6000);
                log.resend(seq, len);
                for (auto &e : m)
                    if (seq >= e.lo && seq < e.hi)
                    {
                        e.hi = seq + len;
                        if (e.at >= 0)
                            e.at = ~e.at;
                        break;
                    }
            }
            else if (high > una)
            {
                una += g() % (high - una + 1);
                log.acked(una, op);
                while (!m.empty() && m[0].hi <= una)
                    m.erase(m.begin());
            }
            if (S.h_n != m.size())
            {
                printf("rtt history trial %d op %d: %u entries, model %zu\n", trial, op, S.h_n, m.size());
                return 1;
            }
            for (uint32_t j = 0; j < S.h_n; j++)
            {
                const uint32_t x = (S.h_head + j) % cap;
                if (lo[x] != m[j].lo || hi[x] != m[j].hi || at[x] != m[j].at)
                {
                    printf("rtt history trial %d op %d: entry %u differs\n", trial, op, j);
                    return 1;
                }
            }
        }
    }
    puts("rtt history: all agree");
    return 0;
}
