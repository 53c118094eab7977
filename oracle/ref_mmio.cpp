// Test infrastructure: the Matrix Market header of the reference's weight
// files, written and read through the reference's own NIST routines
// (external/nist/mmio.cpp), as RBFFD::writeToAsciiFile / writeToBinaryFile
// (src/rbffd/rbffd.cpp:1283-1296) and loadFromAsciiFile / loadFromBinaryFile
// (rbffd.cpp:995-1005) use them.  Built from the reference sources in place by
// oracle/build.py into oracle/_ref/.
#include <cstdio>
#include "mmio.h"

// Banner and size line of a weight file (the entries follow in the caller's form).
extern "C" int ref_mm_write_header(const char* path, int M, int N, int nz)
{
    FILE* f = fopen(path, "w");
    if (!f) return -1;
    MM_typecode matcode;
    mm_initialize_typecode(&matcode);
    mm_set_matrix(&matcode);
    mm_set_coordinate(&matcode);
    mm_set_real(&matcode);
    mm_write_banner(f, matcode);  // returns nonzero even when it wrote the line
    int rc = mm_write_mtx_crd_size(f, M, N, nz);
    fclose(f);
    return rc;
}

// Read the header; *offset is the byte offset of the first entry.
extern "C" int ref_mm_read_header(const char* path, int* M, int* N, int* nz, long* offset)
{
    FILE* f = fopen(path, "r");
    if (!f) return -1;
    MM_typecode matcode;
    int rc = mm_read_banner(f, &matcode);
    if (rc == 0 && !(mm_is_matrix(matcode) && mm_is_coordinate(matcode) && mm_is_real(matcode))) rc = -2;
    if (rc == 0) rc = mm_read_mtx_crd_size(f, M, N, nz);
    *offset = ftell(f);
    fclose(f);
    return rc;
}
