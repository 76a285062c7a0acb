// Drives the mixed-degree tuner's file format (theeggman.jl_b200/csrc/egg_tunecache.h): records
// written by one process are read back by the next, merged per key, and a malformed file is
// ignored.  Prints "ok" on success.  argv[1]: a scratch directory.
#include <cstdio>
#include <string>

#include "egg_tunecache.h"

static int fails = 0;
#define CHECK(c)                                                  \
    do {                                                          \
        if (!(c)) {                                               \
            std::printf("FAIL line %d: %s\n", __LINE__, #c);      \
            ++fails;                                              \
        }                                                         \
    } while (0)

int main(int argc, char **argv)
{
    const std::string path = std::string(argv[1]) + "/sub/dir/mix_tuning.json";
    egg::TuneRecord a{"NVIDIA B200", 148, 24, 1, 0, 0, 64};
    egg::TuneRecord b{"NVIDIA B200", 148, 32, 1, 0, 0, 32};
    egg::TuneRecord c{"Other GPU", 132, 24, 1, 0, 1, 16};
    CHECK(egg::tune_merge_file(path, a));  // creates the directories
    CHECK(egg::tune_merge_file(path, b));
    CHECK(egg::tune_merge_file(path, c));
    std::vector<egg::TuneRecord> rs;
    CHECK(egg::tune_read_file(path, rs));
    CHECK(rs.size() == 3);
    // A new choice for an existing key replaces it.
    egg::TuneRecord a2 = a;
    a2.batched = 1;
    a2.group = 16;
    CHECK(egg::tune_merge_file(path, a2));
    CHECK(egg::tune_read_file(path, rs));
    CHECK(rs.size() == 3);
    bool found = false;
    for (const auto &r : rs)
        if (r.same_key(a)) found = r.batched == 1 && r.group == 16;
    CHECK(found);
    CHECK(rs[2].device == "Other GPU" && rs[2].sms == 132);
    // The same degree tuned on a batch of another size class is another record.
    egg::TuneRecord a3 = a;
    a3.size = 4;
    a3.group = 32;
    CHECK(egg::tune_merge_file(path, a3));
    CHECK(egg::tune_read_file(path, rs));
    CHECK(rs.size() == 4);
    found = false;
    for (const auto &r : rs)
        if (r.same_key(a3)) found = r.group == 32 && r.size == 4;
    CHECK(found);
    // Malformed text is refused; a missing file reads as empty.
    std::vector<egg::TuneRecord> bad;
    CHECK(!egg::tune_parse("{\"format\": 1, \"entries\": [{\"device\": \"x\", \"K\": 2}]}", bad));
    CHECK(!egg::tune_parse("not json", bad));
    // A record without "size" (the first format) is refused, so such a file is tuned again.
    CHECK(!egg::tune_parse("{\"format\": 1, \"entries\": [{\"device\": \"x\", \"sms\": 1, \"K\": 24, "
                           "\"dtype\": 1, \"prec\": 0, \"batched\": 0, \"group\": 64}]}",
                           bad));
    CHECK(!egg::tune_read_file(std::string(argv[1]) + "/missing.json", bad) && bad.empty());
    if (fails == 0) std::printf("ok\n");
    return fails ? 1 : 0;
}
