// rmb_oracle_cli.cpp -- `rmblastn`-compatible command line over the CPU oracle
// (TEST INFRASTRUCTURE).  Restates rmblastn/src/main.rs:516-770 for the single-chunk
// tabular path: same option names and defaults, outfmt 6 only.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "rmb_oracle.hpp"

using namespace rmbo;

int main(int argc, char** argv) {
    try {
        std::string db, query, matrix, outfmt = "6 score";
        Params p;
        p.dust = true;
        p.word_size = 11;
        int threads = 1;
        int mask_level = -1;
        bool stats = false;
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            // NCBI spellings: single dash and underscores (main.rs:64-101)
            if (a.size() > 1 && a[0] == '-' && a[1] != '-') a = "-" + a;
            for (auto& c : a)
                if (c == '_') c = '-';
            auto val = [&]() -> std::string {
                if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
                return argv[++i];
            };
            if (a == "--db") db = val();
            else if (a == "--query") query = val();
            else if (a == "--matrix") matrix = val();
            else if (a == "--gapopen") p.gap_open = std::stoi(val());
            else if (a == "--gapextend") p.gap_extend = std::stoi(val());
            else if (a == "--word-size") p.word_size = std::stoi(val());
            else if (a == "--xdrop-ungap") p.xdrop_ungap = std::stoi(val());
            else if (a == "--xdrop-gap") p.xdrop_gap = std::stoi(val());
            else if (a == "--xdrop-gap-final") p.xdrop_gap_final = std::stoi(val());
            else if (a == "--min-raw-gapped-score") p.min_raw_gapped_score = std::stoi(val());
            else if (a == "--complexity-adjust") p.complexity_adjust = true;
            else if (a == "--dust") {
                std::string d = val();
                if (d == "yes" || d == "true") p.dust = true;
                else if (d == "no" || d == "false") p.dust = false;
                else throw std::runtime_error("--dust expects yes or no");
            } else if (a == "--mask-level") mask_level = std::stoi(val());
            else if (a == "--outfmt") outfmt = val();
            else if (a == "--num-threads") threads = std::stoi(val());
            else if (a == "--mt-mode") val();
            else if (a == "--stats") stats = true;
            else if (a == "--evalue") p.evalue = std::stod(val());
            else if (a == "--matrix-lambda") p.cli_stats[0] = std::stod(val());
            else if (a == "--matrix-k") p.cli_stats[1] = std::stod(val());
            else if (a == "--matrix-alpha") p.cli_stats[2] = std::stod(val());
            else if (a == "--matrix-beta") p.cli_stats[3] = std::stod(val());
            else throw std::runtime_error("unknown option " + a);
        }
        if (matrix.empty()) throw std::runtime_error("--matrix is required");
        p.mask_level = mask_level < 0 ? 101u : (uint32_t)mask_level;
        std::istringstream fs(outfmt);
        std::string t;
        std::vector<std::string> fields;
        fs >> t;
        if (t != "6") throw std::runtime_error("only -outfmt 6 is supported");
        while (fs >> t) fields.push_back(t);
        Matrix m = load_matrix(matrix);
        p.matrix_name = matrix;
        std::vector<Subject> subjects;
        if (db.size() > 5 && db.substr(db.size() - 5) == ".2bit") subjects = read_twobit(db);
        else
            for (auto& r : read_fasta(db)) subjects.push_back(make_subject(r.id, r.seq));
        auto queries = read_fasta(query);
        Counters ctr;
        auto t0 = std::chrono::steady_clock::now();
        std::string out;
        for (auto& q : queries) {
            auto res = search_query(q.seq, q.id, subjects, p, m, threads, stats ? &ctr : nullptr);
            for (auto& r : res) {
                out += format_tabular(r, fields);
                out.push_back('\n');
            }
        }
        fwrite(out.data(), 1, out.size(), stdout);
        if (stats) {
            double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            fprintf(stderr,
                    "STATS seconds=%.3f word_hits=%llu seeds=%llu ungapped=%llu prelim_dp=%llu prelims=%llu tb_dp=%llu "
                    "finals=%llu so_cells=%llu tb_cells=%llu\n",
                    s, (unsigned long long)ctr.word_hits, (unsigned long long)ctr.seeds,
                    (unsigned long long)ctr.ungapped, (unsigned long long)ctr.prelim_dp,
                    (unsigned long long)ctr.prelims, (unsigned long long)ctr.tb_dp, (unsigned long long)ctr.finals,
                    (unsigned long long)ctr.so_cells, (unsigned long long)ctr.tb_cells);
        }
        return 0;
    } catch (const std::exception& e) {
        fprintf(stderr, "Error: %s\n", e.what());
        return 1;
    }
}
