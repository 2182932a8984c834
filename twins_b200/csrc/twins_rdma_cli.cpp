// twins-rdma: the reference's RDMA command line (src/rdma/rmain.cu:1-42, 1023-1240) over the
// twins-b200 C ABI.
//   twins-rdma CONFIG --topo=F --flows=F [--out=fct.txt] [--rate=100Gbps] [--delay=1000] [--q3cap=4096]
//              [--txtrace=F [--from=ns] [--until=ns] [--txcap=N]] [KEY=VALUE ...]
//   twins-rdma CONFIG --batch=JOBFILE --outdir=DIR [--path=DIR:DIR...] [options] [KEY=VALUE ...]
// CONFIG: an HPCC config file ("KEY v1 v2 ..." per line); KEY=VALUE (KEY=V1,V2,.. for several
// values) overrides it. A job file's lines "name topo flows [KEY=VALUE ...]" are worlds of one batch
// (their overrides on top of CONFIG's and the command line's), run side by side; world name's
// results go to DIR/name.fct. Topologies: "hosts H / switches S / link A B", every link at --rate
// with --delay ns. Flow files: src,dst,flow_size,start_ns (lines that do not parse are skipped).
// Output: "id start_ns fct_ns" per completed flow, by id; stdout: the flows done and simulated time,
// and the counters line, as the reference prints them. Exit status: 0 every flow done; 2 some
// unfinished at the stop time; 3 an error counter (an overflow: the results are not exact); 1 a
// usage, input or device error.
// --txtrace: every transmission starting in [--from, --until] (ns), one per line "ns node dev kind
// src dst sport seq bytes ecn" sorted by (ns, node, dev), kind one of D A N P R (the reference's
// format, src/rdma/rmain.cu:2262-2282; one world only). --txcap: records kept (default 64 Mi, as
// the reference keeps).
// --q3cap: frames a switch port's data queue holds (an overflow is reported, exit 3). The reference's
// launch-shape options (--win, --gwin, --rank*, --persist, --spread, --serial, --tail, --dcap) change
// no result; they are accepted and have no effect here.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/twinsb200.h"

namespace
{

typedef std::map<std::string, std::vector<std::string>> Config;

bool read_text(const std::string &path, std::string &out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        return false;
    std::stringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

bool read_config(const std::string &path, Config &cfg)
{
    std::string text;
    if (!read_text(path, text))
        return false;
    std::istringstream lines(text);
    std::string line;
    while (std::getline(lines, line))
    {
        std::istringstream is(line);
        std::string key, v;
        if (!(is >> key))
            continue;
        std::vector<std::string> vals;
        while (is >> v)
            vals.push_back(v);
        cfg[key] = vals;
    }
    return true;
}

// KEY=V or KEY=V1,V2,...
void set_override(Config &cfg, const std::string &k, const std::string &v)
{
    std::vector<std::string> vals;
    size_t b = 0;
    for (size_t c; (c = v.find(',', b)) != std::string::npos; b = c + 1)
        vals.push_back(v.substr(b, c - b));
    vals.push_back(v.substr(b));
    cfg[k] = vals;
}

std::string config_text(const Config &cfg)
{
    std::string t;
    for (auto &kv : cfg)
    {
        t += kv.first;
        for (auto &v : kv.second)
            t += " " + v;
        t += "\n";
    }
    return t;
}

// ns-3 DataRate strings: a number and a unit (bps, Kbps, Mbps, Gbps; b/s, Kb/s, Mb/s, Gb/s)
unsigned long long parse_rate(const std::string &s)
{
    size_t i = 0;
    while (i < s.size() && (isdigit((unsigned char)s[i]) || s[i] == '.'))
        i++;
    const double v = atof(s.substr(0, i).c_str());
    const char u = i < s.size() ? s[i] : 0;
    const double m = u == 'K' || u == 'k' ? 1e3 : u == 'M' ? 1e6 : u == 'G' ? 1e9 : 1;
    return (unsigned long long)(v * m);
}

struct Flows
{
    std::vector<int> src, dst;
    std::vector<long long> size, start;
};

bool load_flows(const std::string &path, Flows &f)
{
    std::string text;
    if (!read_text(path, text))
        return false;
    std::istringstream lines(text);
    std::string line;
    while (std::getline(lines, line))
    {
        long long a, b;
        unsigned long long sz, st;
        if (sscanf(line.c_str(), "%lld,%lld,%llu,%llu", &a, &b, &sz, &st) != 4)
            continue;
        f.src.push_back((int)a);
        f.dst.push_back((int)b);
        f.size.push_back((long long)sz);
        f.start.push_back((long long)st);
    }
    return true;
}

struct Job
{
    std::string name, topo, flows;
    Config cfg;
};

} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        fprintf(stderr, "usage: twins-rdma CONFIG --topo=F --flows=F --out=F [KEY=VALUE ...]\n"
                        "       twins-rdma CONFIG --batch=JOBFILE --outdir=DIR [KEY=VALUE ...]\n");
        return 1;
    }
    Config base;
    if (!read_config(argv[1], base))
    {
        fprintf(stderr, "cannot open %s\n", argv[1]);
        return 1;
    }
    std::string topo_file, flow_file, out_file = "fct.txt", batch_file, out_dir = ".", data_dirs, rate_s = "100Gbps", tx_file;
    long long delay = 1000, tx_from = 0, tx_until = LLONG_MAX, tx_cap = 64ll << 20;
    int device = 0, q3cap = 4096;
    for (int i = 2; i < argc; i++)
    {
        const std::string a = argv[i];
        const size_t eq = a.find('=');
        const std::string k = a.substr(0, eq), v = eq == std::string::npos ? "" : a.substr(eq + 1);
        if (k == "--topo")
            topo_file = v;
        else if (k == "--flows")
            flow_file = v;
        else if (k == "--out")
            out_file = v;
        else if (k == "--batch")
            batch_file = v;
        else if (k == "--outdir")
            out_dir = v;
        else if (k == "--path")
            data_dirs = v;
        else if (k == "--rate")
            rate_s = v;
        else if (k == "--delay")
            delay = atoll(v.c_str());
        else if (k == "--device")
            device = atoi(v.c_str());
        else if (k == "--q3cap")
            q3cap = atoi(v.c_str());
        else if (k == "--txtrace")
            tx_file = v;
        else if (k == "--from")
            tx_from = atoll(v.c_str());
        else if (k == "--until")
            tx_until = atoll(v.c_str());
        else if (k == "--txcap")
            tx_cap = atoll(v.c_str());
        else if (k == "--win" || k == "--gwin" || k == "--rank" || k == "--rank-join" || k == "--rank-bs" || k == "--rank-every" ||
                 k == "--persist" || k == "--spread" || k == "--serial" || k == "--tail" || k == "--tail-auto" || k == "--dcap")
            continue; // (launch shapes and capacities of the reference's kernels: no result depends on them)
        else if (k.compare(0, 2, "--") != 0 && eq != std::string::npos)
            set_override(base, k, v);
        else
        {
            fprintf(stderr, "unknown argument %s\n", argv[i]);
            return 1;
        }
    }
    const unsigned long long bps = parse_rate(rate_s);
    auto find_file = [&](const std::string &f) {
        size_t b = 0;
        while (!data_dirs.empty() && b <= data_dirs.size())
        {
            const size_t c = data_dirs.find(':', b);
            const std::string p = data_dirs.substr(b, c == std::string::npos ? std::string::npos : c - b) + "/" + f;
            if (std::ifstream(p))
                return p;
            if (c == std::string::npos)
                break;
            b = c + 1;
        }
        return f;
    };
    std::vector<Job> jobs;
    if (batch_file.empty())
        jobs.push_back({"run", topo_file, flow_file, base});
    else
    {
        std::string text;
        if (!read_text(batch_file, text))
        {
            fprintf(stderr, "cannot open %s\n", batch_file.c_str());
            return 1;
        }
        std::istringstream lines(text);
        std::string line;
        while (std::getline(lines, line))
        {
            std::istringstream is(line);
            Job j;
            std::string kv;
            if (!(is >> j.name) || j.name[0] == '#' || !(is >> j.topo >> j.flows))
                continue;
            j.cfg = base;
            while (is >> kv)
            {
                const size_t eq = kv.find('=');
                if (eq == std::string::npos)
                {
                    fprintf(stderr, "%s: bad override %s\n", j.name.c_str(), kv.c_str());
                    return 1;
                }
                set_override(j.cfg, kv.substr(0, eq), kv.substr(eq + 1));
            }
            j.topo = find_file(j.topo);
            j.flows = find_file(j.flows);
            jobs.push_back(j);
        }
        if (jobs.empty())
        {
            fprintf(stderr, "%s: no jobs\n", batch_file.c_str());
            return 1;
        }
    }
    tb_ctx *ctx = nullptr;
    if (tb_ctx_create(device, 0, &ctx))
    {
        fprintf(stderr, "%s\n", tb_last_error());
        return 1;
    }
    if (tb_rdma_set_queue_cap(ctx, q3cap))
    {
        fprintf(stderr, "%s\n", tb_last_error());
        return 1;
    }
    if (!tx_file.empty())
    {
        if (!batch_file.empty())
        {
            fprintf(stderr, "--txtrace traces one world (no --batch)\n");
            return 1;
        }
        if (tb_rdma_set_txtrace(ctx, tx_cap, tx_from, tx_until))
        {
            fprintf(stderr, "%s\n", tb_last_error());
            return 1;
        }
    }
    std::vector<Flows> flows(jobs.size());
    int F = 0;
    for (size_t i = 0; i < jobs.size(); i++)
    {
        std::string topo;
        if (!read_text(jobs[i].topo, topo))
        {
            fprintf(stderr, "cannot open %s\n", jobs[i].topo.c_str());
            return 1;
        }
        if (!load_flows(jobs[i].flows, flows[i]))
        {
            fprintf(stderr, "cannot open %s\n", jobs[i].flows.c_str());
            return 1;
        }
        const Flows &f = flows[i];
        int w = 0;
        if (tb_world_add_rdma(ctx, config_text(jobs[i].cfg).c_str(), topo.c_str(), (int)f.src.size(), f.src.data(), f.dst.data(),
                              f.size.data(), f.start.data(), bps, delay, &w))
        {
            fprintf(stderr, "%s: %s\n", jobs[i].name.c_str(), tb_last_error());
            return 1;
        }
        F += (int)f.src.size();
    }
    if (jobs.size() > 1)
        printf("%zu worlds, %d flows\n", jobs.size(), F);
    const auto t0 = std::chrono::steady_clock::now();
    const int status = tb_run(ctx, 0);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (status < 0)
    {
        fprintf(stderr, "%s\n", tb_last_error());
        return 1;
    }
    unsigned done = 0;
    for (size_t i = 0; i < jobs.size(); i++)
    {
        const size_t n = flows[i].src.size();
        std::vector<long long> start(n), fct(n);
        tb_rdma_results(ctx, (int)i, start.data(), fct.data());
        const std::string path = batch_file.empty() ? out_file : out_dir + "/" + jobs[i].name + ".fct";
        FILE *fo = fopen(path.c_str(), "w");
        if (!fo)
        {
            fprintf(stderr, "cannot write %s\n", path.c_str());
            return 1;
        }
        for (size_t j = 0; j < n; j++)
            if (fct[j] >= 0)
            {
                fprintf(fo, "%zu %lld %lld\n", j, start[j], fct[j]);
                done++;
            }
        fclose(fo);
    }
    unsigned long long ev[40] = {};
    tb_counters(ctx, 0, ev, 40);
    tb_stats st{};
    tb_get_stats(ctx, &st);
    printf("flows done %u of %d; simulated %.6f s in %.3f s wall (%lld launches)\n", done, F, (double)st.slots * delay * 1e-9, wall, st.launches);
    printf("drops %llu marks %llu pauses %llu resumes %llu nacks %llu | undecided ties %llu, on lost tails %llu | overflows: tx %llu queue "
           "%llu ackq %llu qps %llu due %llu | acks for done QPs %llu\n",
           ev[0], ev[1], ev[2], ev[3], ev[11], ev[8], ev[9], ev[4], ev[5], ev[6], ev[7], ev[12], ev[10]);
    if (!tx_file.empty())
    {
        long long n = 0, total = 0;
        tb_rdma_txtrace(ctx, nullptr, 0, &n, &total);
        std::vector<tb_tx_record> rec((size_t)std::min(total, tx_cap));
        tb_rdma_txtrace(ctx, rec.data(), (long long)rec.size(), &n, &total);
        if (total > (long long)rec.size())
            fprintf(stderr, "txtrace: %lld records, %zu kept\n", total, rec.size());
        FILE *ft = fopen(tx_file.c_str(), "w");
        if (!ft)
        {
            fprintf(stderr, "cannot write %s\n", tx_file.c_str());
            return 1;
        }
        const char kinds[] = "DANPR";
        for (long long i = 0; i < n; i++)
        {
            const tb_tx_record &x = rec[(size_t)i];
            fprintf(ft, "%lld %d %d %c %u %u %u %u %u %u\n", x.ts_ns, x.node, x.dev, x.kind < 5 ? kinds[x.kind] : '?', x.a, x.b, x.sport, x.seq,
                    (unsigned)x.size, (unsigned)x.ecn);
        }
        fclose(ft);
    }
    const bool bad = ev[4] || ev[5] || ev[6] || ev[7] || ev[12];
    if (bad)
        fprintf(stderr, "warning: capacity overflow, results are not exact\n");
    if (ev[13])
        fprintf(stderr, "warning: %llu data frames reached receivers after their flows' last byte; if their senders had completed, "
                        "ns-3 would answer them with NACKs (not modelled)\n", ev[13]);
    if (ev[8] || ev[9])
        fprintf(stderr, "warning: ties the chains did not decide exactly (%llu undecided, %llu on lost tails)\n", ev[8], ev[9]);
    tb_ctx_destroy(ctx);
    return bad ? 3 : done == (unsigned)F ? 0 : 2;
}
