// Drives GpuSkipSequentialScan (include/tremor_b200_sss.hpp) exactly as the reference's
// tremor_main drives SkipSequentialScan (tremor_main.cpp:754-790): build from a waveform
// file, then search_knn and search_threshold writing the reference's CSV files.
//   sss_drop_in <waveform.bin> <samples> <m> <queries.bin> <count> <k> <merge> <corr> <out>
// writes <out>.knn.csv and <out>.thr_0.csv.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "tremor_b200_sss.hpp"

int main(int argc, char **argv)
{
    if (argc != 10)
    {
        std::fprintf(stderr, "usage: %s waveform samples m queries count k merge corr out\n", argv[0]);
        return 2;
    }
    const unsigned long long samples = std::strtoull(argv[2], nullptr, 10);
    const int m = std::atoi(argv[3]), count = std::atoi(argv[5]), k = std::atoi(argv[6]);
    const int merge = std::atoi(argv[7]);
    const float corr = std::strtof(argv[8], nullptr);
    const std::string out = argv[9];
    std::vector<float> queries(static_cast<size_t>(count) * m);
    FILE *f = std::fopen(argv[4], "rb");
    if (f == nullptr || std::fread(queries.data(), sizeof(float), queries.size(), f) != queries.size())
        return 3;
    std::fclose(f);
    try
    {
        GpuSkipSequentialScan scan(1, 8, merge, 0, false);
        scan.build(argv[1], samples, m);
        scan.search_knn(queries.data(), count, k, out + ".knn.csv");
        scan.search_threshold(queries.data(), count, corr, out + ".thr");
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
