// tremor_b200_cli: the reference's external-data driver (tremor_main.cpp) with the exact
// scan on the GPU. Same options, inputs (raw float32 files), validation, output files
// (kNN CSV "tID, k, pos, corr"; threshold shard "<output>_0.csv" with "Query, Counter,
// Position, Cross Correlation") and timings CSV (node_rank,index_time,query_time,index_gb),
// one node. Every --method (tremor, skip-sequential, sequential, gpu-scan) returns the same
// exact answers, so all of them run the GPU scan; options that tune the reference's index
// or its MPI groups are accepted and validated as it does, then have no effect.
//
//   tremor_b200_cli --dataset data.bin --queries q.bin --window-length 1024 [--mode knn]
//                   [--k 10] [--threshold 0.93] [--merge-offset 0] [--output out.csv] ...
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "tremor_b200_sss.hpp"

namespace
{

struct Options
{
    std::string dataset_path, queries_path, output_path, benchmark_output_path;
    bool dataset_size_set = false, query_count_set = false, skip_benchmark_report = false;
    uint64_t dataset_size = 0, query_count = 0, window_length = 0;
    bool knn = true;
    uint64_t knn_k = 10, threshold_result_slots = 1;
    float threshold_correlation = 0.93f;
    int search_workers = 4, index_threads = 4, leaf_size = 2000, paa_segments = 16, replication_groups = 0;
    int pq_threshold_divisor = 16, merge_offset = 0, device = 0;
    std::string method = "tremor", refinement = "leaf";
    double scan_fallback_fraction = 0.01;
    bool verbose = false, print_knn_results = false;
    uint64_t print_query_limit = 5;
};

struct HelpRequested
{
};

void usage(const char *program)
{
    std::printf(
        "Usage: %s --dataset FILE --queries FILE --window-length N [options]\n"
        "  --mode knn|threshold        search mode (default knn)\n"
        "  --k N                       neighbours per query (default 10)\n"
        "  --threshold C               correlation threshold (default 0.93)\n"
        "  --merge-offset N            exclusion zone / threshold merge (default 0)\n"
        "  --dataset-size N            samples to use (default: the whole file)\n"
        "  --query-count N             queries to use (default: the whole file)\n"
        "  --output PATH               kNN CSV / threshold shard prefix\n"
        "  --benchmark-output PATH     timings CSV (default <output>.timings.csv)\n"
        "  --no-benchmark-report       write no timings CSV\n"
        "  --method tremor|skip-sequential|sequential|gpu-scan   (all run the exact GPU scan)\n"
        "  --device N                  GPU (default 0)\n"
        "  --print-knn-results, --print-query-limit N, --verbose\n"
        "  accepted for compatibility: --scan-fallback-fraction, --refinement, --threshold-result-slots,\n"
        "    --search-workers, --query-threads, --index-threads, --leaf-size, --paa-segments,\n"
        "    --replication-groups, --pq-threshold-divisor\n",
        program);
}

const char *value(int argc, char **argv, int &i, const std::string &arg)
{
    if (i + 1 >= argc)
        throw std::invalid_argument("Missing value for " + arg);
    return argv[++i];
}

uint64_t parse_u64(const std::string &v, const std::string &option)
{
    size_t used = 0;
    unsigned long long r = 0;
    try
    {
        if (!v.empty() && v[0] == '-')
            throw std::invalid_argument("negative");
        r = std::stoull(v, &used);
    }
    catch (const std::exception &)
    {
        throw std::invalid_argument("Invalid unsigned integer for " + option + ": " + v);
    }
    if (used != v.size())
        throw std::invalid_argument("Invalid unsigned integer for " + option + ": " + v);
    return r;
}

int parse_int(const std::string &v, const std::string &option)
{
    size_t used = 0;
    long long r = 0;
    try
    {
        r = std::stoll(v, &used);
    }
    catch (const std::exception &)
    {
        throw std::invalid_argument("Invalid integer for " + option + ": " + v);
    }
    if (used != v.size() || r > std::numeric_limits<int>::max() || r < std::numeric_limits<int>::min())
        throw std::invalid_argument("Invalid integer for " + option + ": " + v);
    return static_cast<int>(r);
}

float parse_float(const std::string &v, const std::string &option)
{
    size_t used = 0;
    float r = 0.0f;
    try
    {
        r = std::stof(v, &used);
    }
    catch (const std::exception &)
    {
        throw std::invalid_argument("Invalid float for " + option + ": " + v);
    }
    if (used != v.size() || !std::isfinite(r))
        throw std::invalid_argument("Invalid float for " + option + ": " + v);
    return r;
}

Options parse(int argc, char **argv)
{
    Options o;
    for (int i = 1; i < argc; i++)
    {
        const std::string a = argv[i];
        if (a == "--help" || a == "-h")
            throw HelpRequested{};
        else if (a == "--dataset")
            o.dataset_path = value(argc, argv, i, a);
        else if (a == "--queries")
            o.queries_path = value(argc, argv, i, a);
        else if (a == "--output")
            o.output_path = value(argc, argv, i, a);
        else if (a == "--benchmark-output")
            o.benchmark_output_path = value(argc, argv, i, a);
        else if (a == "--no-benchmark-report")
            o.skip_benchmark_report = true;
        else if (a == "--dataset-size")
        {
            o.dataset_size = parse_u64(value(argc, argv, i, a), a);
            o.dataset_size_set = true;
        }
        else if (a == "--query-count")
        {
            o.query_count = parse_u64(value(argc, argv, i, a), a);
            o.query_count_set = true;
        }
        else if (a == "--window-length")
            o.window_length = parse_u64(value(argc, argv, i, a), a);
        else if (a == "--mode")
        {
            const std::string m = value(argc, argv, i, a);
            if (m == "knn" || m == "KNN")
                o.knn = true;
            else if (m == "threshold" || m == "THRESHOLD")
                o.knn = false;
            else
                throw std::invalid_argument("Unknown --mode: " + m);
        }
        else if (a == "--method")
        {
            o.method = value(argc, argv, i, a);
            if (o.method != "tremor" && o.method != "skip-sequential" && o.method != "sequential" &&
                o.method != "gpu-scan")
                throw std::invalid_argument("Unknown --method: " + o.method +
                                            " (expected tremor, skip-sequential, sequential or gpu-scan)");
        }
        else if (a == "--scan-fallback-fraction")
        {
            o.scan_fallback_fraction = std::stod(value(argc, argv, i, a));
            if (std::isnan(o.scan_fallback_fraction))
                throw std::invalid_argument("--scan-fallback-fraction must be a number");
        }
        else if (a == "--refinement")
            o.refinement = value(argc, argv, i, a);
        else if (a == "--k")
            o.knn_k = parse_u64(value(argc, argv, i, a), a);
        else if (a == "--threshold")
            o.threshold_correlation = parse_float(value(argc, argv, i, a), a);
        else if (a == "--threshold-result-slots")
            o.threshold_result_slots = parse_u64(value(argc, argv, i, a), a);
        else if (a == "--search-workers" || a == "--query-threads")
            o.search_workers = parse_int(value(argc, argv, i, a), a);
        else if (a == "--index-threads")
            o.index_threads = parse_int(value(argc, argv, i, a), a);
        else if (a == "--leaf-size")
            o.leaf_size = parse_int(value(argc, argv, i, a), a);
        else if (a == "--paa-segments")
            o.paa_segments = parse_int(value(argc, argv, i, a), a);
        else if (a == "--replication-groups")
            o.replication_groups = parse_int(value(argc, argv, i, a), a);
        else if (a == "--pq-threshold-divisor")
            o.pq_threshold_divisor = parse_int(value(argc, argv, i, a), a);
        else if (a == "--merge-offset")
            o.merge_offset = parse_int(value(argc, argv, i, a), a);
        else if (a == "--device")
            o.device = parse_int(value(argc, argv, i, a), a);
        else if (a == "--verbose")
            o.verbose = true;
        else if (a == "--print-knn-results")
            o.print_knn_results = true;
        else if (a == "--print-query-limit")
            o.print_query_limit = parse_u64(value(argc, argv, i, a), a);
        else
            throw std::invalid_argument("Unknown argument: " + a);
    }
    // the reference's checks (tremor_main.cpp:374-456)
    if (o.dataset_path.empty())
        throw std::invalid_argument("--dataset is required");
    if (o.queries_path.empty())
        throw std::invalid_argument("--queries is required");
    if (o.window_length == 0)
        throw std::invalid_argument("--window-length must be greater than 0");
    if (o.window_length % 8 != 0)
        throw std::invalid_argument("--window-length must be divisible by 8");
    if (o.paa_segments <= 0)
        throw std::invalid_argument("--paa-segments must be greater than 0");
    if (o.window_length % static_cast<uint64_t>(o.paa_segments) != 0)
        throw std::invalid_argument("--window-length must be divisible by --paa-segments");
    if (o.dataset_size_set && o.dataset_size < o.window_length)
        throw std::invalid_argument("--dataset-size must be at least --window-length");
    if (o.query_count_set && o.query_count == 0)
        throw std::invalid_argument("--query-count must be greater than 0");
    if (o.knn_k == 0)
        throw std::invalid_argument("--k must be greater than 0");
    if (o.threshold_result_slots == 0)
        throw std::invalid_argument("--threshold-result-slots must be greater than 0");
    if (o.threshold_correlation < -1.0f || o.threshold_correlation > 1.0f)
        throw std::invalid_argument("--threshold must be between -1.0 and 1.0");
    if (o.search_workers <= 0 || o.index_threads <= 0)
        throw std::invalid_argument("thread counts must be greater than 0");
    if (o.leaf_size <= 0)
        throw std::invalid_argument("--leaf-size must be greater than 0");
    if (o.pq_threshold_divisor <= 0)
        throw std::invalid_argument("--pq-threshold-divisor must be greater than 0");
    if (o.merge_offset < 0)
        throw std::invalid_argument("--merge-offset must be non-negative");
    if (o.replication_groups < 0)
        throw std::invalid_argument("--replication-groups must be non-negative");
    if (o.window_length > static_cast<uint64_t>(std::numeric_limits<int>::max()))
        throw std::invalid_argument("--window-length is too large for this TREMOR build");
    if (o.knn_k > static_cast<uint64_t>(std::numeric_limits<int>::max()))
        throw std::invalid_argument("requested result count is too large for this TREMOR build");
    if (o.output_path.empty())
        o.output_path = o.knn ? "tremor_knn.csv" : "tremor_threshold";
    if (o.benchmark_output_path.empty() && !o.skip_benchmark_report)
        o.benchmark_output_path = o.output_path + ".timings.csv";
    return o;
}

uint64_t float_count(const std::string &path)
{
    struct stat st;
    if (stat(path.c_str(), &st) != 0)
        throw std::runtime_error("cannot stat " + path + ": " + std::strerror(errno));
    return static_cast<uint64_t>(st.st_size) / sizeof(float);
}

// Reads `count` floats from the start of a file, in chunks (the reference reads its rank's
// chunk of the record, Tremor.cpp:214-262).
std::vector<float> read_floats(const std::string &path, uint64_t count)
{
    std::vector<float> out(count);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (f == nullptr)
        throw std::runtime_error("cannot open " + path + ": " + std::strerror(errno));
    const uint64_t chunk = 1ull << 24;
    for (uint64_t at = 0; at < count; at += chunk)
    {
        const size_t want = static_cast<size_t>(std::min(chunk, count - at));
        if (std::fread(out.data() + at, sizeof(float), want, f) != want)
        {
            std::fclose(f);
            throw std::runtime_error("short read from " + path);
        }
    }
    std::fclose(f);
    return out;
}

void write_timings(const std::string &path, double index_s, double query_s, double index_gb)
{
    if (path.empty())
        return;
    FILE *out = std::fopen(path.c_str(), "w");
    if (out == nullptr)
    {
        std::fprintf(stderr, "Warning: cannot open benchmark report file %s: %s\n", path.c_str(), std::strerror(errno));
        return;
    }
    std::fprintf(out, "node_rank,index_time,query_time,index_gb\n");
    std::fprintf(out, "%zu,%0.6f,%0.6f,%0.3f\n", static_cast<size_t>(0), index_s, query_s, index_gb);
    std::fclose(out);
    std::printf("Benchmark timings CSV: %s\n", path.c_str());
}

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace

int main(int argc, char **argv)
{
    Options o;
    try
    {
        o = parse(argc, argv);
    }
    catch (const HelpRequested &)
    {
        usage(argv[0]);
        return 0;
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "Error: %s\n", e.what());
        usage(argv[0]);
        return 2;
    }
    try
    {
        const auto input_t0 = std::chrono::steady_clock::now();
        const uint64_t file_floats = float_count(o.dataset_path);
        const uint64_t n = o.dataset_size_set ? o.dataset_size : file_floats;
        if (n > file_floats)
            throw std::runtime_error("--dataset-size exceeds float count in " + o.dataset_path);
        if (n < o.window_length)
            throw std::runtime_error("dataset has fewer samples than --window-length");
        const uint64_t query_floats = float_count(o.queries_path);
        uint64_t qc = o.query_count;
        if (o.query_count_set)
        {
            if (qc * o.window_length > query_floats)
                throw std::runtime_error("--query-count * --window-length exceeds float count in " + o.queries_path);
        }
        else
        {
            if (query_floats % o.window_length != 0)
                throw std::runtime_error("query file float count is not divisible by --window-length");
            qc = query_floats / o.window_length;
            if (qc == 0)
                throw std::runtime_error("query file contains no complete query vectors");
        }
        if (qc > static_cast<uint64_t>(std::numeric_limits<int>::max()))
            throw std::runtime_error("query count is too large for this TREMOR build");
        const std::vector<float> queries = read_floats(o.queries_path, qc * o.window_length);
        const std::vector<float> raw = read_floats(o.dataset_path, n);
        const double input_s = seconds_since(input_t0);
        const int m = static_cast<int>(o.window_length);

        std::printf("\nTREMOR external-data run (GPU scan)\n");
        std::printf("  mode: %s\n", o.knn ? "knn" : "threshold");
        std::printf("  dataset: %s\n", o.dataset_path.c_str());
        std::printf("  dataset_size: %llu float32 samples\n", static_cast<unsigned long long>(n));
        std::printf("  queries: %s\n", o.queries_path.c_str());
        std::printf("  query_count: %llu\n", static_cast<unsigned long long>(qc));
        std::printf("  window_length: %d\n", m);
        std::printf("  output: %s\n", o.output_path.c_str());
        if (o.knn)
            std::printf("  k: %llu\n", static_cast<unsigned long long>(o.knn_k));
        else
            std::printf("  threshold_correlation: %0.6f\n", o.threshold_correlation);
        std::printf("  merge_offset: %d\n", o.merge_offset);
        std::printf("  method: %s (exact scan on GPU %d)\n", o.method.c_str(), o.device);

        GpuSkipSequentialScan scan(o.search_workers, o.paa_segments, o.merge_offset, o.replication_groups,
                                   o.method != "sequential", o.device);
        const auto build_t0 = std::chrono::steady_clock::now();
        scan.build(raw.data(), n, m);
        const double index_s = seconds_since(build_t0);
        const auto search_t0 = std::chrono::steady_clock::now();
        if (o.knn)
        {
            std::vector<uint64_t> I;
            std::vector<float> D;
            scan.search_knn(queries.data(), static_cast<int>(qc), static_cast<int>(o.knn_k), o.output_path, &I, &D);
            if (o.print_knn_results)
            {
                const uint64_t show = std::min<uint64_t>(qc, o.print_query_limit);
                std::printf("\nKNN search preview\n");
                for (uint64_t q = 0; q < show; q++)
                {
                    std::printf("  query %llu\n", static_cast<unsigned long long>(q));
                    for (uint64_t k = 0; k < o.knn_k; k++)
                    {
                        const size_t at = static_cast<size_t>(q * o.knn_k + k);
                        std::printf("    #%llu: offset=%llu squared_ed=%0.6f corr=%0.6f\n",
                                    static_cast<unsigned long long>(k + 1), static_cast<unsigned long long>(I[at]),
                                    D[at], tm_ed_to_cc(D[at], m));
                    }
                }
            }
        }
        else
            scan.search_threshold(queries.data(), static_cast<int>(qc), o.threshold_correlation, o.output_path);
        const double query_s = input_s + seconds_since(search_t0);
        if (!o.skip_benchmark_report)
            write_timings(o.benchmark_output_path, index_s, query_s, scan.summary_memory_bytes() / 1e9);
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "Error: %s\n", e.what());
        return 1;
    }
    return 0;
}
