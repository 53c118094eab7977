// Weight files in the reference's Matrix Market formats
// (RBFFD::writeToAsciiFile / writeToBinaryFile, src/rbffd/rbffd.cpp:1265-1375;
// RBFFD::loadFromAsciiFile / loadFromBinaryFile, rbffd.cpp:983-1210), so that
// weights move between the reference's CPU path and this library both ways.
//
// Both forms start with the text header the reference writes through the NIST
// mmio routines (external/nist/mmio.cpp): the banner line
// "%%MatrixMarket matrix coordinate real general" and the size line
// "M N nz" (stencils, nodes, weights).  Then one entry per stencil weight, in
// stencil order: the 1-based row (the stencil's centre) and column (the
// stencil node) and the weight -- as text "%d %d %24.16le" (17 significant
// digits: every double reads back exactly), or in the binary form as raw
// native int, int, double records directly after the header.  Reading
// follows the reference: entries fill a row's weights in file order; in
// addition every entry's column is checked against the stencil, so weights
// written for other stencils are refused instead of misapplied.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/rbffd_sm100.h"

namespace {

const char* BANNER = "%%MatrixMarket";

bool valid_sizes(int N, int n_pad, const int* st, const int* st_len)
{
    if (N <= 0 || n_pad <= 0 || !st) return false;
    if (st_len)
        for (int i = 0; i < N; i++)
            if (st_len[i] < 1 || st_len[i] > n_pad) return false;
    return true;
}

int row_len(const int* st_len, int n_pad, int i) { return st_len ? st_len[i] : n_pad; }

// Banner and size line; false on anything but a real general coordinate matrix.
bool read_header(FILE* f, long long* M, long long* Ncol, long long* nz)
{
    char line[1100];
    if (!fgets(line, sizeof line, f)) return false;
    char b[64], obj[64], fmt[64], type[64], sym[64];
    if (sscanf(line, "%63s %63s %63s %63s %63s", b, obj, fmt, type, sym) != 5) return false;
    if (strcmp(b, BANNER) != 0) return false;
    for (char* s : {obj, fmt, type, sym})
        for (char* c = s; *c; c++) *c = (char)tolower((unsigned char)*c);
    if (strcmp(obj, "matrix") || strcmp(fmt, "coordinate") || strcmp(type, "real") || strcmp(sym, "general"))
        return false;
    do {  // comment lines, as mm_read_mtx_crd_size skips them
        if (!fgets(line, sizeof line, f)) return false;
    } while (line[0] == '%');
    return sscanf(line, "%lld %lld %lld", M, Ncol, nz) == 3;
}

}  // namespace

extern "C" int rbffd_weights_file_write(const char* filename, int binary, int N, int n_pad, const int* st,
                                        const int* st_len, const double* w)
{
    if (!filename || !w || !valid_sizes(N, n_pad, st, st_len)) return RBFFD_ERR_INVALID;
    long long nz = 0;
    for (int i = 0; i < N; i++) nz += row_len(st_len, n_pad, i);
    if (nz > 2147483647ll) return RBFFD_ERR_UNSUPPORTED;  // the format's counts are int
    FILE* f = fopen(filename, "wb");
    if (!f) return RBFFD_ERR_INVALID;
    bool ok = fprintf(f, "%s matrix coordinate real general\n", BANNER) > 0;
    ok = ok && fprintf(f, "%d %d %lld\n", N, N, nz) > 0;  // one rank: stencils x nodes, square
    for (int i = 0; i < N && ok; i++) {
        const int* s = st + (size_t)i * n_pad;
        const int row = s[0] + 1;  // the stencil's centre, 1-based
        for (int j = 0; j < row_len(st_len, n_pad, i) && ok; j++) {
            const int col = s[j] + 1;
            const double v = w[(size_t)i * n_pad + j];
            if (binary) {
                ok = fwrite(&row, sizeof(int), 1, f) == 1 && fwrite(&col, sizeof(int), 1, f) == 1 &&
                     fwrite(&v, sizeof(double), 1, f) == 1;
            } else {
                ok = fprintf(f, "%d %d %24.16le\n", row, col, v) > 0;
            }
        }
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? RBFFD_OK : RBFFD_ERR_INVALID;
}

extern "C" int rbffd_weights_file_read(const char* filename, int binary, int N, int n_pad, const int* st,
                                       const int* st_len, double* w)
{
    if (!filename || !w || !valid_sizes(N, n_pad, st, st_len)) return RBFFD_ERR_INVALID;
    FILE* f = fopen(filename, "rb");
    if (!f) return RBFFD_ERR_INVALID;
    long long M = 0, Ncol = 0, nz = 0, expected = 0;
    for (int i = 0; i < N; i++) expected += row_len(st_len, n_pad, i);
    if (!read_header(f, &M, &Ncol, &nz) || M != N || nz != expected) {
        fclose(f);
        return RBFFD_ERR_INVALID;
    }
    memset(w, 0, sizeof(double) * (size_t)N * n_pad);
    std::vector<int> filled(N, 0);
    int rc = RBFFD_OK, cur = -1, j = 0;
    for (long long e = 0; e < nz && rc == RBFFD_OK; e++) {
        int I, J;
        double v;
        if (binary) {
            if (fread(&I, sizeof(int), 1, f) != 1 || fread(&J, sizeof(int), 1, f) != 1 ||
                fread(&v, sizeof(double), 1, f) != 1) {
                rc = RBFFD_ERR_INVALID;
                break;
            }
        } else if (fscanf(f, "%d %d %le", &I, &J, &v) != 3) {
            rc = RBFFD_ERR_INVALID;
            break;
        }
        I--, J--;
        if (I < 0 || I >= N || J < 0) {
            rc = RBFFD_ERR_INVALID;
            break;
        }
        if (I != cur) {  // entries of a row are consecutive, in stencil order
            cur = I;
            j = 0;
        }
        if (j >= row_len(st_len, n_pad, I) || st[(size_t)I * n_pad + j] != J || filled[I] != j) {
            rc = RBFFD_ERR_INVALID;  // not this grid's stencil
            break;
        }
        w[(size_t)I * n_pad + j] = v;
        filled[I] = ++j;
    }
    fclose(f);
    if (rc == RBFFD_OK)
        for (int i = 0; i < N; i++)
            if (filled[i] != row_len(st_len, n_pad, i)) return RBFFD_ERR_INVALID;
    return rc;
}
