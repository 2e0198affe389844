// rmb_oracle_stats.cpp -- Karlin-Altschul E-values and bit scores (TEST INFRASTRUCTURE).
// Restates rmblast-lib/src/ka_stats.rs:153-300 (default mode, without the ALP fit) and
// rmblast-stats/rmstats/src: rmblast_tables.rs:26-75, eff_lengths.rs, length_adjust.rs,
// evalue.rs, and the NCBI tabular renderings of rmblast-lib/src/output.rs:244-289.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <strings.h>

#include "rmb_oracle.hpp"

namespace rmbo {

namespace {
// rmstats tables_data.rs RMBLAST_MATRIX_KA: (matrix file name, gap open, gap extend, lambda, K, H)
struct StatRow { const char* name; int go, ge; double lambda, k, h; };
const StatRow STATS[] = {
    {"14p35g.matrix", 29, 6, 0.1241860392, 0.2565118357, 0.3349210581}, {"14p37g.matrix", 29, 6, 0.1243509013, 0.2538327145, 0.3484386549},
    {"14p39g.matrix", 29, 6, 0.118108197, 0.2381799563, 0.3209988017}, {"14p41g.matrix", 29, 6, 0.1209164962, 0.251696198, 0.3474870514},
    {"14p43g.matrix", 29, 6, 0.1204338701, 0.2484920137, 0.3397421893}, {"14p45g.matrix", 29, 6, 0.1281012415, 0.2651519027, 0.3664022073},
    {"14p47g.matrix", 29, 6, 0.116957149, 0.2334091021, 0.3226817428}, {"14p49g.matrix", 29, 6, 0.1167697593, 0.2289233061, 0.3136272703},
    {"14p51g.matrix", 29, 6, 0.1238779017, 0.2467119379, 0.32413383}, {"14p53g.matrix", 29, 6, 0.1211022467, 0.2307304663, 0.2949314272},
    {"18p35g.matrix", 28, 5, 0.120477663, 0.2111410357, 0.2484902185}, {"18p37g.matrix", 28, 5, 0.1213800379, 0.2057492194, 0.2637651575},
    {"18p39g.matrix", 28, 5, 0.1228853168, 0.2111281814, 0.2802003038}, {"18p41g.matrix", 28, 5, 0.1096830298, 0.1715966796, 0.2171487218},
    {"18p43g.matrix", 28, 5, 0.1179924113, 0.1957371364, 0.2544060456}, {"18p45g.matrix", 28, 5, 0.1184247414, 0.2068045787, 0.2641082233},
    {"18p47g.matrix", 28, 5, 0.115878332, 0.1842046578, 0.2407688057}, {"18p49g.matrix", 28, 5, 0.1248964218, 0.2141853759, 0.2675489103},
    {"18p51g.matrix", 28, 5, 0.1106793836, 0.1621592148, 0.1979815532}, {"18p53g.matrix", 28, 5, 0.1082347513, 0.1408677318, 0.1771724651},
    {"20p35g.matrix", 25, 5, 0.1112832877, 0.1466667286, 0.1741696491}, {"20p37g.matrix", 25, 5, 0.1134511409, 0.1501236494, 0.193180875},
    {"20p39g.matrix", 25, 5, 0.1233401001, 0.1853070864, 0.2324952723}, {"20p41g.matrix", 25, 5, 0.1088138918, 0.1409300313, 0.1778018484},
    {"20p43g.matrix", 25, 5, 0.1097495426, 0.1408421343, 0.1813610542}, {"20p45g.matrix", 25, 5, 0.1101110565, 0.1402262486, 0.1803401526},
    {"20p47g.matrix", 25, 5, 0.1198508511, 0.175230183, 0.2232474228}, {"20p49g.matrix", 25, 5, 0.1150022018, 0.1500562415, 0.1891763921},
    {"20p51g.matrix", 25, 5, 0.1101356126, 0.1310353805, 0.1457676446}, {"20p53g.matrix", 25, 5, 0.1239625969, 0.1752022586, 0.210665934},
    {"25p35g.matrix", 22, 5, 0.0965155465, 0.0677355511, 0.0964040436}, {"25p37g.matrix", 22, 5, 0.0989264764, 0.076371967, 0.1025772304},
    {"25p39g.matrix", 22, 5, 0.1005843197, 0.0805691511, 0.1108913867}, {"25p41g.matrix", 22, 5, 0.1030661339, 0.0840485952, 0.1237017673},
    {"25p43g.matrix", 22, 5, 0.115543436, 0.1226554129, 0.1495157932}, {"25p45g.matrix", 22, 5, 0.0973402625, 0.074202019, 0.1029029688},
    {"25p47g.matrix", 22, 5, 0.0967346256, 0.0743885008, 0.0995494785}, {"25p49g.matrix", 22, 5, 0.1070577141, 0.0941947942, 0.1181023643},
    {"25p51g.matrix", 22, 5, 0.1044972455, 0.0789036639, 0.1081508568}, {"25p53g.matrix", 22, 5, 0.0977828435, 0.0607500307, 0.0834178835},
    {"30p53g.matrix", 22, 5, 0.1204393447, 0.1065198197, 0.1243912966}, {"comparison.matrix", 20, 5, 0.09836223, 0.0789918084, 0.1116129577},
};
}  // namespace

// ka_stats.rs:153-300 resolve (StatsMode::Default) + kbp_for_recipe + the alpha/beta choice of
// eff_lengths.rs:40-70.
KaStats resolve_stats(const std::string& matrix_name, int go, int ge, const double cli[4], const Matrix& m) {
    KaStats s;
    std::string base = matrix_name;
    const size_t sl = base.find_last_of('/');
    if (sl != std::string::npos) base = base.substr(sl + 1);
    const bool cli_set = cli[0] > 0.0 && cli[1] > 0.0 && cli[2] > 0.0;  // MatrixCliOverrides::is_set
    for (const StatRow& r : STATS) {
        if (r.go == go && r.ge == ge && strcasecmp(r.name, base.c_str()) == 0) {
            s = KaStats{r.lambda, r.k, std::log(r.k), r.h, cli_set ? cli[2] : r.lambda / r.h, cli_set ? cli[3] : 0.0, 1};
            return s;
        }
    }
    auto cli_like = [&](double lambda, double k, double alpha, double beta, int src) {
        return KaStats{lambda, k, std::log(k), lambda / alpha, alpha, beta, src};
    };
    if (cli_set) return cli_like(cli[0], cli[1], cli[2], cli[3], 2);
    if (m.has_karlin) {
        const double* kc = m.karlin;  // lambda, K, H, alpha, beta
        const double alpha = kc[3] > 0.0 ? kc[3] : kc[2] > 0.0 ? kc[0] / kc[2] : 0.0;
        if (kc[0] > 0.0 && kc[1] > 0.0 && alpha > 0.0) return cli_like(kc[0], kc[1], alpha, kc[4], 3);
    }
    return s;  // sentinel
}

// length_adjust.rs compute_length_adjustment (BLAST_ComputeLengthAdjustment)
int32_t length_adjustment(double k, double log_k, double alpha_d_lambda, double beta, int32_t query_length,
                          int64_t db_length, int32_t db_num_seqs, bool* converged_out) {
    const int kMax = 20;
    const double m = query_length, n = (double)db_length, bn = db_num_seqs;
    double ell_min = 0.0, ell_max = 0.0, ell_next = 0.0;
    bool converged = false;
    const double a = bn, mb = m * bn + n, c = n * m - std::max(m, n) / k;
    if (c < 0.0) {
        if (converged_out) *converged_out = false;
        return 0;
    }
    ell_max = 2.0 * c / (mb + std::sqrt(mb * mb - 4.0 * a * c));
    for (int i = 1; i <= kMax; ++i) {
        const double ell = ell_next;
        const double ss = (m - ell) * (n - bn * ell);
        const double ell_bar = alpha_d_lambda * (log_k + std::log(ss)) + beta;
        if (ell_bar >= ell) {
            ell_min = ell;
            if (ell_bar - ell_min <= 1.0) { converged = true; break; }
            if (ell_min == ell_max) break;
        } else {
            ell_max = ell;
        }
        if (ell_min <= ell_bar && ell_bar <= ell_max) ell_next = ell_bar;
        else ell_next = (i == 1) ? ell_max : (ell_min + ell_max) / 2.0;
    }
    int32_t la = (int32_t)ell_min;
    if (converged) {
        const double ell = std::ceil(ell_min);
        if (ell <= ell_max) {
            const double ss = (m - ell) * (n - bn * ell);
            if (alpha_d_lambda * (log_k + std::log(ss)) + beta >= ell) la = (int32_t)ell;
        }
    }
    if (converged_out) *converged_out = converged;
    return la;
}

// eff_lengths.rs calc_eff_lengths_custom_matrix: the effective search space (0 without stats)
int64_t effective_search_space(const KaStats& s, int32_t query_length, int64_t db_length, int32_t db_num_seqs) {
    if (query_length <= 0 || s.lambda <= 0.0) return 0;
    const int32_t la =
        length_adjustment(s.k, s.log_k, s.alpha / s.lambda, s.beta, query_length, db_length, db_num_seqs, nullptr);
    int64_t eff_db = db_length - (int64_t)db_num_seqs * (int64_t)la;
    if (eff_db <= 0) eff_db = 1;
    return eff_db * (int64_t)(query_length - la);
}

// evalue.rs hsp_evalue (round_down false on this path) and hsp_bit_score
double evalue_of(int32_t score, const KaStats& s, int64_t searchsp) {
    if (s.lambda <= 0.0) return 1.0;
    if (s.lambda < 0.0 || s.k < 0.0 || s.h < 0.0) return -1.0;
    return (double)searchsp * std::exp(-s.lambda * (double)score + s.log_k);
}
double bitscore_of(int32_t score, const KaStats& s) {
    if (s.lambda <= 0.0) return 0.0;
    return ((double)score * s.lambda - s.log_k) / 0.69314718055994530942;
}

// output.rs:244-289 format_evalue / format_bit_score
std::string format_evalue(double e) {
    char b[64];
    if (e < 1.0e-180) return "0.0";
    if (e < 0.0009) snprintf(b, sizeof b, "%.2e", e);
    else if (e < 0.1) snprintf(b, sizeof b, "%.3f", e);
    else if (e < 1.0) snprintf(b, sizeof b, "%.2f", e);
    else if (e < 10.0) snprintf(b, sizeof b, "%.1f", e);
    else snprintf(b, sizeof b, "%.0f", e);
    return b;
}
std::string format_bitscore(double v) {
    char b[64];
    if (v > 99999.0) snprintf(b, sizeof b, "%.3e", v);
    else if (v > 99.9) snprintf(b, sizeof b, "%3ld", (long)v);
    else snprintf(b, sizeof b, "%4.1f", v);
    return b;
}

}  // namespace rmbo
