/*
 * Link-time probe around run_bndiag_wrapper for the reference's C example.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  The reference's
 * src/c_interface/libnegf_c_example.c is compiled unchanged and linked with
 * -Wl,--wrap=run_bndiag_wrapper, so its call lands here first; this passes it
 * on to libnegf_b200.so's run_bndiag_wrapper and, when NEGF_C_EXAMPLE_DUMP
 * names a directory, writes the CSC input and the returned CSC band there as
 * raw arrays (in.bin / out.bin: three int32 counts m, n, nnz, then colptr,
 * rowval, nzval) for the parity test to check against the oracle.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int32_t m, n, nnz;
  int32_t* colptr;
  int32_t* rowval;
  void* nzval;
} Csc;

Csc __real_run_bndiag_wrapper(int32_t m, int32_t n, int32_t nnz_in, int32_t* colptr_in, int32_t* rowval_in,
                              void* nzval_in, int32_t n_blocks, int32_t* block_sizes_in, int32_t n_dict,
                              const char** dict_keys_in, int32_t* dict_vals_in, int32_t is_hermitian);

static void dump(const char* dir, const char* name, int32_t m, int32_t n, int32_t nnz, const int32_t* colptr,
                 const int32_t* rowval, const void* nzval) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* f = fopen(path, "wb");
  if (!f) return;
  const int32_t hdr[3] = {m, n, nnz};
  fwrite(hdr, sizeof(int32_t), 3, f);
  if (colptr) fwrite(colptr, sizeof(int32_t), (size_t)n + 1, f);
  if (rowval) fwrite(rowval, sizeof(int32_t), (size_t)nnz, f);
  if (nzval) fwrite(nzval, 16, (size_t)nnz, f);
  fclose(f);
}

Csc __wrap_run_bndiag_wrapper(int32_t m, int32_t n, int32_t nnz_in, int32_t* colptr_in, int32_t* rowval_in,
                              void* nzval_in, int32_t n_blocks, int32_t* block_sizes_in, int32_t n_dict,
                              const char** dict_keys_in, int32_t* dict_vals_in, int32_t is_hermitian) {
  const char* dir = getenv("NEGF_C_EXAMPLE_DUMP");
  if (dir) {
    dump(dir, "in.bin", m, n, nnz_in, colptr_in, rowval_in, nzval_in);
    char path[4096];
    snprintf(path, sizeof path, "%s/blocks.bin", dir);
    FILE* f = fopen(path, "wb");
    if (f) {
      fwrite(&n_blocks, sizeof(int32_t), 1, f);
      fwrite(block_sizes_in, sizeof(int32_t), (size_t)n_blocks, f);
      fwrite(&is_hermitian, sizeof(int32_t), 1, f);
      fclose(f);
    }
  }
  Csc r = __real_run_bndiag_wrapper(m, n, nnz_in, colptr_in, rowval_in, nzval_in, n_blocks, block_sizes_in, n_dict,
                                    dict_keys_in, dict_vals_in, is_hermitian);
  if (dir) dump(dir, "out.bin", r.m, r.n, r.nnz, r.colptr, r.rowval, r.nzval);
  return r;
}
