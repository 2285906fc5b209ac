// csv.cu -- CSV datasets for the evaluator (host code only).
//
// The reference's two readers (src/Dataset.cpp:83-151), as a C entry point:
//   1-D   (load_csv_1d): the first line is a header; every later non-empty
//         line with a comma gives x (text before the first comma) and y
//         (text after it); lines without a comma are skipped.
//   multi (load_csv_multi): the first line is a header; every later
//         non-empty line is split at every comma; all columns but the last
//         are features, the last is the target.
// Numbers are read like std::stof: leading spaces skipped, the longest
// numeric prefix converted, an error when nothing converts or the value is
// out of float range.  The reference throws in those cases; this reader
// returns GALOP_E_INVALID with the line number.  A row whose column count
// differs from the first data row is an error here (the reference reads
// past the row).  ss_tot is the reference's two-pass total sum of squares
// of the targets (src/Dataset.cpp:35-47).
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/galop_b200.h"
#include "context.cuh"

namespace {

void set_err(char* err, int32_t err_len, const std::string& msg) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", msg.c_str());
}

// std::stof semantics on one field.
bool read_float(const std::string& field, float* out) {
    const char* s = field.c_str();
    char* end = nullptr;
    errno = 0;
    const float v = std::strtof(s, &end);
    if (end == s || errno == ERANGE) return false;
    *out = v;
    return true;
}

}  // namespace

extern "C" {

int galop_csv_read(const char* path, int32_t multi, galop_csv_dataset* out, char* err, int32_t err_len) {
    if (!path || !out) return GALOP_E_INVALID;
    std::memset(out, 0, sizeof *out);
    std::ifstream f(path);
    if (!f) {
        set_err(err, err_len, std::string("cannot open ") + path);
        return GALOP_E_INVALID;
    }
    std::string line;
    std::getline(f, line);   // header
    std::vector<float> xs, ys;
    int64_t cols = -1, lineno = 1;
    while (std::getline(f, line)) {
        ++lineno;
        if (line.empty()) continue;
        if (!multi) {
            const size_t comma = line.find(',');
            if (comma == std::string::npos) continue;
            float x, y;
            if (!read_float(line.substr(0, comma), &x) || !read_float(line.substr(comma + 1), &y)) {
                set_err(err, err_len, std::string(path) + ":" + std::to_string(lineno) + ": not a float pair");
                return GALOP_E_INVALID;
            }
            xs.push_back(x);
            ys.push_back(y);
            continue;
        }
        std::vector<float> row;
        size_t start = 0;
        for (;;) {
            const size_t comma = line.find(',', start);
            const size_t stop = comma == std::string::npos ? line.size() : comma;
            float v;
            if (!read_float(line.substr(start, stop - start), &v)) {
                set_err(err, err_len, std::string(path) + ":" + std::to_string(lineno) + ": field " +
                                          std::to_string(row.size() + 1) + " is not a float");
                return GALOP_E_INVALID;
            }
            row.push_back(v);
            if (comma == std::string::npos) break;
            start = comma + 1;
        }
        if (cols < 0) {
            cols = (int64_t)row.size();
            if (cols < 2) {
                set_err(err, err_len, std::string(path) + ": a multi-feature csv needs >= 2 columns");
                return GALOP_E_INVALID;
            }
        } else if ((int64_t)row.size() != cols) {
            set_err(err, err_len, std::string(path) + ":" + std::to_string(lineno) + ": " +
                                      std::to_string(row.size()) + " columns, expected " + std::to_string(cols));
            return GALOP_E_INVALID;
        }
        xs.insert(xs.end(), row.begin(), row.end() - 1);
        ys.push_back(row.back());
    }
    if (multi && cols < 0) {
        set_err(err, err_len, std::string(path) + ": no data rows");
        return GALOP_E_INVALID;
    }
    const int64_t n = (int64_t)ys.size();
    out->n_cases = n;
    out->num_inputs = multi ? (int32_t)(cols - 1) : 1;
    out->inputs = (float*)std::malloc(std::max<size_t>(xs.size(), 1) * sizeof(float));
    out->targets = (float*)std::malloc(std::max<size_t>(ys.size(), 1) * sizeof(float));
    if (!out->inputs || !out->targets) {
        galop_csv_free(out);
        return GALOP_E_NOMEM;
    }
    if (!xs.empty()) std::memcpy(out->inputs, xs.data(), xs.size() * sizeof(float));
    if (!ys.empty()) std::memcpy(out->targets, ys.data(), ys.size() * sizeof(float));
    out->ss_tot = targets_ss_tot(out->targets, n);
    return GALOP_OK;
}

void galop_csv_free(galop_csv_dataset* d) {
    if (!d) return;
    std::free(d->inputs);
    std::free(d->targets);
    d->inputs = nullptr;
    d->targets = nullptr;
}

}  // extern "C"
