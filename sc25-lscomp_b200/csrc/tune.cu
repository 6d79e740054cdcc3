// tune.cu -- the launch-configuration tuner: the table of measured choices
// (process-wide), its text form, and the C ABI that controls it
// (include/lscomp.h, lscomp_tune_*).
//
// A configuration is the encoder CTA shape (compute groups x warps per group)
// and the tile size in blocks; for the decoder only the tile size.  Every
// configuration writes the same stream (the stream format knows nothing of
// tiles), so a call may run with any of them; the tuner times the
// candidates on the call's own buffers the first time a key is seen and
// keeps the fastest.  The timing loop itself is a template in codec_host.h
// (tune_choose), since it launches the typed kernels.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include "codec_host.h"

namespace lsc_host {
namespace {

struct Entry {
    TuneCfg cfg;
    std::vector<std::pair<TuneCfg, float>> times;  // ms per call of each candidate, when measured here
};

struct KeyLess {
    bool operator()(const TuneKey &a, const TuneKey &b) const
    {
        return std::make_tuple(a.es, a.layout, a.pool, a.kind, a.vec, a.bzb) <
               std::make_tuple(b.es, b.layout, b.pool, b.kind, b.vec, b.bzb);
    }
};

std::mutex g_mu;
std::map<TuneKey, Entry, KeyLess> g_table;
uint64_t g_hits = 0;  // calls that found their key in the table
int g_mode = -1;  // -1: not read from the environment yet

int mode_locked()
{
    if (g_mode < 0) {
        const char *e = getenv("LSCOMP_AUTOTUNE");
        g_mode = (e && e[0] == '0') ? 0 : 1;
    }
    return g_mode;
}

bool valid_cfg(const TuneKey &k, const TuneCfg &c)
{
    const uint32_t maxb = k.es == 2 ? 256u : 128u;
    if (c.tile_blocks < 8 || c.tile_blocks > maxb || c.tile_blocks % 8) return false;
    if (c.shape < -1 || c.shape > 3) return false;
    if (c.shape >= 1 && k.es != 2) return false;
    if (c.shape == 2 && k.kind == kTuneBatch) return false;  // 2 x 13 runs single stacks only
    // 2 x 8 with the short paths: lossless single-stack compression only
    if (c.shape == 3 && (k.kind != kTuneCompress || k.layout != BINS_IDENT)) return false;
    if (k.vec != 16 && k.vec != 4 && !(k.vec == 2 && k.es == 2)) return false;
    return k.es == 2 || k.es == 4;
}

void format_entry(std::string &s, const TuneKey &k, const Entry &e)
{
    char line[256];
    snprintf(line, sizeof line, "%u %u %u %u %u %u -> %d %u", k.es, k.layout, k.pool, k.kind, k.vec, k.bzb,
             e.cfg.shape, e.cfg.tile_blocks);
    s += line;
    for (const auto &t : e.times) {
        snprintf(line, sizeof line, " | %d %u %.4f", t.first.shape, t.first.tile_blocks, t.second);
        s += line;
    }
    s += '\n';
}

}  // namespace

int tune_mode()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return mode_locked();
}

bool tune_lookup(const TuneKey &k, TuneCfg &c)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find(k);
    if (it == g_table.end()) return false;
    c = it->second.cfg;
    g_hits++;
    return true;
}

void tune_store(const TuneKey &k, const TuneCfg &c, const std::vector<std::pair<TuneCfg, float>> &times)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Entry &e = g_table[k];
    e.cfg = c;
    e.times = times;
}

// Candidates per element size, call kind and bins layout.  Encoder: CTA
// shape 2 x 8, 2 x 7 or (single stacks) 2 x 13 warps (uint16), and for
// lossless uint16 single stacks 2 x 8 with the short paths for small values;
// tiles of up to 256 or 128 blocks (uint16; 128 or 64 for uint32).
// Decoder: tiles of 256 or 128 (128 or 64) blocks.
std::vector<TuneCfg> tune_candidates(int es, int kind, int layout)
{
    const uint32_t big = es == 2 ? 256u : 128u, small = big / 2;
    std::vector<TuneCfg> v;
    if (kind == kTuneDecompress) {
        v.push_back({-1, big});
        v.push_back({-1, small});
        return v;
    }
    v.push_back({0, big});
    if (es == 2) v.push_back({1, big});
    if (es == 2 && kind == kTuneCompress) v.push_back({2, big});
    if (es == 2 && kind == kTuneCompress && layout == BINS_IDENT) v.push_back({3, big});
    v.push_back({0, small});
    if (es == 2) v.push_back({1, small});
    return v;
}

}  // namespace lsc_host

using namespace lsc_host;

extern "C" {

int lscomp_tune_mode(int mode)
{
    std::lock_guard<std::mutex> lk(g_mu);
    const int prev = mode_locked();
    if (mode == 0 || mode == 1) g_mode = mode;
    return prev;
}

uint64_t lscomp_tune_hits(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_hits;
}

int lscomp_tune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_table.clear();
    return LSCOMP_OK;
}

uint64_t lscomp_tune_report(char *buf, uint64_t cap)
{
    std::string s;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (const auto &kv : g_table) format_entry(s, kv.first, kv.second);
    }
    if (buf && cap) {
        const size_t n = s.size() < cap - 1 ? s.size() : (size_t)(cap - 1);
        memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return (uint64_t)s.size() + 1;
}

int lscomp_tune_save(const char *path)
{
    if (!path) return LSCOMP_ERR_ARG;
    std::string s;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (const auto &kv : g_table) format_entry(s, kv.first, kv.second);
    }
    FILE *f = fopen(path, "w");
    if (!f) return LSCOMP_ERR_ARG;
    const bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
    return (fclose(f) == 0 && ok) ? LSCOMP_OK : LSCOMP_ERR_ARG;
}

int lscomp_tune_load(const char *path)
{
    if (!path) return LSCOMP_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return LSCOMP_ERR_ARG;
    std::vector<std::pair<TuneKey, TuneCfg>> got;
    char line[4096];
    int st = LSCOMP_OK;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '\n' || line[0] == '#') continue;
        unsigned es, layout, pool, kind, vec, bzb, tb;
        int shape;
        if (sscanf(line, "%u %u %u %u %u %u -> %d %u", &es, &layout, &pool, &kind, &vec, &bzb, &shape, &tb) != 8) {
            st = LSCOMP_ERR_ARG;
            break;
        }
        TuneKey k{(uint8_t)es, (uint8_t)layout, (uint8_t)pool, (uint8_t)kind, (uint8_t)vec, bzb};
        TuneCfg c{shape, tb};
        if (layout > 3 || pool > 1 || kind > 2 || !valid_cfg(k, c)) {
            st = LSCOMP_ERR_ARG;
            break;
        }
        got.push_back({k, c});
    }
    fclose(f);
    if (st) return st;  // a malformed file changes nothing
    std::lock_guard<std::mutex> lk(g_mu);
    for (const auto &kc : got) {
        Entry &e = g_table[kc.first];
        e.cfg = kc.second;
        e.times.clear();
    }
    return LSCOMP_OK;
}

}  // extern "C"
