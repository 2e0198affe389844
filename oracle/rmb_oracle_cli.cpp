// rmb_oracle_cli.cpp -- `rmblastn`-compatible command line over the CPU oracle
// (TEST INFRASTRUCTURE).  Restates rmblastn/src/main.rs:516-770 for the single-chunk
// tabular path and pairwise output (outfmt 0, the default): same option names and defaults.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include <fstream>
#include <map>
#include <set>

#include "rmb_oracle.hpp"

using namespace rmbo;

int main(int argc, char** argv) {
    try {
        std::string db, query, matrix, outfmt = "0", gilist;
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
            else if (a == "--gilist") gilist = val();
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
        const bool pairwise = t == "0";
        if (t != "6" && !pairwise) throw std::runtime_error("only -outfmt 6 and 0 are supported");
        while (fs >> t) fields.push_back(t);
        Matrix m = load_matrix(matrix);
        p.matrix_name = matrix;
        std::vector<Subject> subjects;
        std::map<std::string, std::string> deflines;
        const bool twobit = db.size() > 5 && db.substr(db.size() - 5) == ".2bit";
        if (twobit) subjects = read_twobit(db);
        else
            for (auto& r : read_fasta(db)) {
                deflines[r.id] = r.defline;
                subjects.push_back(make_subject(r.id, r.seq));
            }
        if (!gilist.empty()) {  // main.rs:1444-1470: keep the listed ids (a bare number also names "gi|n")
            std::ifstream gf(gilist);
            if (!gf) throw std::runtime_error("opening gilist '" + gilist + "'");
            std::set<std::string> keep;
            std::string ln;
            while (std::getline(gf, ln)) {
                size_t a = ln.find_first_not_of(" \t\r\n"), b = ln.find_last_not_of(" \t\r\n");
                if (a == std::string::npos) continue;
                std::string e = ln.substr(a, b - a + 1);
                if (e.find_first_not_of("0123456789") == std::string::npos) keep.insert("gi|" + e);
                keep.insert(e);
            }
            std::vector<Subject> kept;
            for (auto& s : subjects)
                if (keep.count(s.id)) kept.push_back(std::move(s));
            subjects.swap(kept);
        }
        auto queries = read_fasta(query);
        Counters ctr;
        auto t0 = std::chrono::steady_clock::now();
        std::string out;
        uint64_t total = 0;
        for (auto& s : subjects) total += s.len();
        if (pairwise) out += pairwise_program_header(db, subjects.size(), total);
        for (auto& q : queries) {
            auto res = search_query(q.seq, q.id, subjects, p, m, threads, stats ? &ctr : nullptr);
            if (pairwise) {
                std::vector<std::pair<size_t, size_t>> mask;  // main.rs:948-956 pairwise_query_mask
                if (p.dust) {
                    std::vector<uint8_t> c = q.seq;
                    mask = dust_mask(c);
                }
                out += pairwise_results(res, q.defline, (uint32_t)(q.seq.size() - 2), twobit ? nullptr : &deflines, mask);
                continue;
            }
            for (auto& r : res) {
                out += format_tabular(r, fields);
                out.push_back('\n');
            }
        }
        if (pairwise) out += pairwise_footer(db, subjects.size(), total, p.gap_open, p.gap_extend);
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
