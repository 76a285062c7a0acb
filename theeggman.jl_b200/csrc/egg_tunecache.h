// egg_tunecache.h -- the mixed-degree batch tuner's choices, kept in a JSON file across processes.
//
// The tuner (egg_mix.cu) times the candidate evaluations of a degree on the first batch that has
// it.  Its choice depends on the GPU model and SM count, the degree, the element type, the
// rounding mode and how many instances of the degree the batch holds (a class: `size` 0..4 for
// fewer than 4, 16, 64, 256 instances, or more), so each record names all of them:
//
//   {"format": 2, "entries": [
//     {"device": "NVIDIA B200", "sms": 148, "K": 24, "dtype": 1, "prec": 0, "size": 4, "batched": 0, "group": 64},
//     ...]}
//
// A process reads the file once, on its first mixed-degree batch, and takes the records of its
// own device; every new choice is merged into the file (all devices' records kept) by writing a
// temporary file and renaming it over the old one, so a reader never sees a partial file.  An
// unreadable or malformed file is ignored (the tuner times again).  Host-only and free of CUDA
// headers, so the format can be exercised without a GPU.
#pragma once

#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace egg {

struct TuneRecord {
    std::string device;
    long long sms = 0, K = 0, dtype = 0, prec = 0, batched = 0, group = 0, size = 0;
    bool same_key(const TuneRecord &o) const
    {
        return device == o.device && sms == o.sms && K == o.K && dtype == o.dtype && prec == o.prec && size == o.size;
    }
};

// Parses the records of a tuning file's text; false if it is not in the format above.
inline bool tune_parse(const std::string &s, std::vector<TuneRecord> &out)
{
    out.clear();
    size_t p = s.find("\"entries\"");
    if (p == std::string::npos) return false;
    p = s.find('[', p);
    if (p == std::string::npos) return false;
    for (;;) {
        const size_t ob = s.find_first_of("{]", p + 1);
        if (ob == std::string::npos) return false;
        if (s[ob] == ']') return true;
        const size_t cb = s.find('}', ob);
        if (cb == std::string::npos) return false;
        const std::string obj = s.substr(ob + 1, cb - ob - 1);
        TuneRecord r;
        int seen = 0;
        size_t q = 0;
        while ((q = obj.find('"', q)) != std::string::npos) {
            const size_t ke = obj.find('"', q + 1);
            if (ke == std::string::npos) return false;
            const std::string key = obj.substr(q + 1, ke - q - 1);
            size_t v = obj.find(':', ke);
            if (v == std::string::npos) return false;
            ++v;
            while (v < obj.size() && obj[v] == ' ') ++v;
            if (v < obj.size() && obj[v] == '"') {
                const size_t ve = obj.find('"', v + 1);
                if (ve == std::string::npos) return false;
                if (key == "device") {
                    r.device = obj.substr(v + 1, ve - v - 1);
                    seen |= 1;
                }
                q = ve + 1;
            } else {
                char *end = nullptr;
                const long long x = std::strtoll(obj.c_str() + v, &end, 10);
                if (end == obj.c_str() + v) return false;
                if (key == "sms") { r.sms = x; seen |= 2; }
                else if (key == "K") { r.K = x; seen |= 4; }
                else if (key == "dtype") { r.dtype = x; seen |= 8; }
                else if (key == "prec") { r.prec = x; seen |= 16; }
                else if (key == "batched") { r.batched = x; seen |= 32; }
                else if (key == "group") { r.group = x; seen |= 64; }
                else if (key == "size") { r.size = x; seen |= 128; }
                q = (size_t)(end - obj.c_str());
            }
        }
        if (seen != 255) return false;  // every field, "size" included (format 1 files are re-tuned)
        out.push_back(r);
        p = cb;
    }
}

inline std::string tune_format(const std::vector<TuneRecord> &rs)
{
    std::string s = "{\"format\": 2, \"entries\": [";
    for (size_t i = 0; i < rs.size(); ++i) {
        const TuneRecord &r = rs[i];
        std::string dev;
        for (char ch : r.device)
            if (ch != '"' && ch != '\\') dev += ch;
        s += i ? ",\n  " : "\n  ";
        s += "{\"device\": \"" + dev + "\", \"sms\": " + std::to_string(r.sms) + ", \"K\": " + std::to_string(r.K) +
             ", \"dtype\": " + std::to_string(r.dtype) + ", \"prec\": " + std::to_string(r.prec) +
             ", \"size\": " + std::to_string(r.size) +
             ", \"batched\": " + std::to_string(r.batched) + ", \"group\": " + std::to_string(r.group) + "}";
    }
    s += "\n]}\n";
    return s;
}

inline bool tune_read_file(const std::string &path, std::vector<TuneRecord> &out)
{
    out.clear();
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::string s;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, n);
    std::fclose(f);
    if (!tune_parse(s, out)) {
        out.clear();
        return false;
    }
    return true;
}

// Merges rec into the file at path (replacing a record of the same key); false on any I/O error.
inline bool tune_merge_file(const std::string &path, const TuneRecord &rec)
{
    std::vector<TuneRecord> rs;
    tune_read_file(path, rs);
    bool replaced = false;
    for (TuneRecord &r : rs)
        if (r.same_key(rec)) {
            r = rec;
            replaced = true;
        }
    if (!replaced) rs.push_back(rec);
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos && slash > 0) {
        // Create the directory chain (mkdir -p) without a shell.
        std::string dir = path.substr(0, slash), acc;
        size_t i = 0;
        while (i <= dir.size()) {
            const size_t j = dir.find('/', i);
            acc = dir.substr(0, j == std::string::npos ? dir.size() : j);
            if (!acc.empty()) ::mkdir(acc.c_str(), 0755);
            if (j == std::string::npos) break;
            i = j + 1;
        }
    }
    const std::string tmp = path + ".tmp" + std::to_string((long long)std::rand());
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    const std::string s = tune_format(rs);
    const bool ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
    if (std::fclose(f) != 0 || !ok) {
        std::remove(tmp.c_str());
        return false;
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        return false;
    }
    return true;
}

// The file the tuner uses: $EGG_TUNE_CACHE when set (an empty value turns the file off), else
// $XDG_CACHE_HOME/eggman_b200/mix_tuning.json, else $HOME/.cache/eggman_b200/mix_tuning.json.
inline std::string tune_cache_path()
{
    if (const char *e = std::getenv("EGG_TUNE_CACHE")) return std::string(e);
    if (const char *x = std::getenv("XDG_CACHE_HOME"))
        if (*x) return std::string(x) + "/eggman_b200/mix_tuning.json";
    if (const char *h = std::getenv("HOME"))
        if (*h) return std::string(h) + "/.cache/eggman_b200/mix_tuning.json";
    return std::string();
}

}  // namespace egg
