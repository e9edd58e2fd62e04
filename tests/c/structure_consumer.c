/* A plain C consumer of the engine's C ABI (include/olfgpu_b200.h), as a cgo / JNI / FFI binding would call it: it
 * reads a packed network (the reference's packed-array layout) from a file, creates the structure, reads its sizes,
 * runs the host check of its block-LU plan, exports its CSR pattern and destroys it.  Host-only entry points: no GPU
 * is needed.  Prints "n nnz buses luBlocks factorLevels violations patternChecksum" on success, exits 1 otherwise.
 *
 * File layout (native-endian int32 / float64): n, nCb, nOb, nSh, nId, then cbParams [nCb*8] f64, cbIndices [nCb*12],
 * obParams [nOb*7] f64, obIndices [nOb*6], shParams [nSh*2] f64, shIndices [nSh*5], identityRows [nId]. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "olfgpu_b200.h"

static void* readAll(FILE* f, size_t bytes) {
    void* p = malloc(bytes > 0 ? bytes : 1);
    if (!p || (bytes > 0 && fread(p, 1, bytes, f) != bytes)) {
        fprintf(stderr, "short read\n");
        exit(1);
    }
    return p;
}

int main(int argc, char** argv) {
    if (argc != 2) return 1;
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 1;
    int32_t head[5];
    if (fread(head, sizeof(int32_t), 5, f) != 5) return 1;
    const int n = head[0], nCb = head[1], nOb = head[2], nSh = head[3], nId = head[4];
    double* cbP = (double*)readAll(f, sizeof(double) * (size_t)nCb * 8);
    int* cbI = (int*)readAll(f, sizeof(int) * (size_t)nCb * 12);
    double* obP = (double*)readAll(f, sizeof(double) * (size_t)nOb * 7);
    int* obI = (int*)readAll(f, sizeof(int) * (size_t)nOb * 6);
    double* shP = (double*)readAll(f, sizeof(double) * (size_t)nSh * 2);
    int* shI = (int*)readAll(f, sizeof(int) * (size_t)nSh * 5);
    int* idr = (int*)readAll(f, sizeof(int) * (size_t)nId);
    fclose(f);

    /* a failing call returns -1 and leaves its reason in olfgpu_last_error */
    if (olfgpu_structure_info(0, NULL, NULL) != -1 || olfgpu_last_error()[0] == '\0') return 1;

    int64_t s = 0;
    if (olfgpu_create_structure(n, nCb, cbP, cbI, nOb, obP, obI, nSh, shP, shI, nId, idr, 19, &s) != 0) {
        fprintf(stderr, "create: %s\n", olfgpu_last_error());
        return 1;
    }
    int info[9];
    int64_t ops = 0;
    int64_t violations = -1;
    char first[256];
    if (olfgpu_structure_info(s, info, &ops) != 0 ||
        olfgpu_structure_check_plan(s, 0, &violations, first, (int)sizeof first) != 0) {
        fprintf(stderr, "query: %s\n", olfgpu_last_error());
        return 1;
    }
    int* rowPtr = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    int* colIdx = (int*)malloc(sizeof(int) * (size_t)info[1]);
    if (olfgpu_structure_export(s, NULL, rowPtr, colIdx, NULL, NULL, NULL, NULL) != 0) return 1;
    long long checksum = 0;
    for (int k = 0; k < info[1]; k++) checksum += (long long)(k % 97 + 1) * colIdx[k];
    for (int r = 0; r <= n; r++) checksum += rowPtr[r];
    if (olfgpu_destroy_structure(s) != 0 || olfgpu_destroy_structure(0) != 0) return 1;
    printf("%d %d %d %d %d %lld %lld\n", info[0], info[1], info[2], info[3], info[4], (long long)violations, checksum);
    free(cbP); free(cbI); free(obP); free(obI); free(shP); free(shI); free(idr); free(rowPtr); free(colIdx);
    return 0;
}
