// sw_params.cu -- scoring matrices from text (the -m option of the
// reference's command line).
//
// The reference documents "-m <str> (Scoring matrix name, default =
// blosum62)" (README.md:130) but its Param parses no such switch and always
// uses the BLOSUM62 table compiled into Param.h:8-51.  Here a matrix can be
// given by name ("blosum62", the built-in table) or as a file in the common
// text layout of substitution matrices: '#' comment lines, one line of column
// letters, then one line per row letter with one integer per column.
#include <cctype>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/swb200.h"
#include "sw_engine.h"

namespace {

// Code of a matrix letter in the search alphabet, or -1 for letters the
// search maps to code 24 (which always scores 0, as -1 does in the
// reference's int8 kernel) and which a matrix therefore cannot score.
int letter_code(char c) {
    static const char* alpha = "ABCDEFGHIKLMNPQRSTVWXYZ";
    const char u = (char)std::toupper((unsigned char)c);
    const char* at = std::strchr(alpha, u);
    if (u && at) return (int)(at - alpha);
    return -1;
}

}  // namespace

extern "C" sw_status sw_params_parse_matrix(sw_params* p, const char* text) {
    if (!p || !text) return swb::thread_fail(SW_ERR_INVALID, "null argument");
    std::istringstream in(text);
    std::string line;
    std::vector<int> cols;
    std::vector<bool> row_seen(24, false);
    int32_t m[32 * 32];
    std::memset(m, 0, sizeof(m));
    int lineno = 0, rows = 0;
    while (std::getline(in, line)) {
        ++lineno;
        const size_t first = line.find_first_not_of(" \t\r");
        if (first == std::string::npos || line[first] == '#') continue;
        std::istringstream ls(line);
        if (cols.empty()) {                       // the column letters
            std::string tok;
            while (ls >> tok) {
                if (tok.size() != 1)
                    return swb::thread_fail(SW_ERR_FORMAT, "line %d: column label '%s' is not one letter",
                                            lineno, tok.c_str());
                cols.push_back(letter_code(tok[0]));
            }
            for (size_t a = 0; a < cols.size(); ++a)
                for (size_t b = a + 1; b < cols.size(); ++b)
                    if (cols[a] >= 0 && cols[a] == cols[b])
                        return swb::thread_fail(SW_ERR_FORMAT, "line %d: column letter repeated", lineno);
            continue;
        }
        std::string lab;
        ls >> lab;
        if (lab.size() != 1)
            return swb::thread_fail(SW_ERR_FORMAT, "line %d: row label '%s' is not one letter", lineno,
                                    lab.c_str());
        const int r = letter_code(lab[0]);
        if (r >= 0) {
            if (row_seen[r]) return swb::thread_fail(SW_ERR_FORMAT, "line %d: row %c repeated", lineno, lab[0]);
            row_seen[r] = true;
        }
        for (size_t k = 0; k < cols.size(); ++k) {
            long v = 0;
            if (!(ls >> v))
                return swb::thread_fail(SW_ERR_FORMAT, "line %d: %zu values for %zu columns", lineno, k,
                                        cols.size());
            if (v < -127 || v > 127)
                return swb::thread_fail(SW_ERR_INVALID, "line %d: score %ld outside -127..127", lineno, v);
            if (r >= 0 && cols[k] >= 0) m[r * 32 + cols[k]] = (int32_t)v;
        }
        std::string extra;
        if (ls >> extra)
            return swb::thread_fail(SW_ERR_FORMAT, "line %d: more values than columns", lineno);
        ++rows;
    }
    if (cols.empty() || rows == 0) return swb::thread_fail(SW_ERR_FORMAT, "no matrix in the text");
    std::memcpy(p->matrix, m, sizeof(m));
    return SW_OK;
}

extern "C" sw_status sw_params_load_matrix(sw_params* p, const char* name_or_path) {
    if (!p || !name_or_path) return swb::thread_fail(SW_ERR_INVALID, "null argument");
    std::string name(name_or_path);
    std::string low = name;
    for (char& c : low) c = (char)std::tolower((unsigned char)c);
    if (low == "blosum62") {
        sw_params d;
        sw_params_default(&d);
        std::memcpy(p->matrix, d.matrix, sizeof(d.matrix));
        return SW_OK;
    }
    FILE* f = std::fopen(name_or_path, "rb");
    if (!f)
        return swb::thread_fail(SW_ERR_INVALID, "no built-in matrix '%s' and no such file",
                                name_or_path);
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
    std::fclose(f);
    return sw_params_parse_matrix(p, text.c_str());
}
