/* Declarations-only stand-in for the cuDSS header, so that the reference's host structure code (which includes it
 * for unrelated members of its structs) compiles on the host.  No function declared here is ever called or linked:
 * the pattern oracle uses only the row-map, pattern and destination builders. */
#pragma once
#include <stdint.h>
#include <stddef.h>
#define CUDSS_VERSION 900
typedef struct cudssContext *cudssHandle_t;
typedef struct cudssConfig *cudssConfig_t;
typedef struct cudssData *cudssData_t;
typedef struct cudssMatrix *cudssMatrix_t;
typedef enum { CUDSS_STATUS_SUCCESS = 0, CUDSS_STATUS_OTHER = 1 } cudssStatus_t;
typedef enum { CUDSS_ALG_DEFAULT = 0, CUDSS_ALG_1, CUDSS_ALG_2, CUDSS_ALG_3, CUDSS_ALG_4, CUDSS_ALG_5 } cudssAlgType_t;
typedef enum { CUDSS_REORDERING_ALG_DEFAULT = 0, CUDSS_REORDERING_ALG_NONE, CUDSS_REORDERING_ALG_AMD,
               CUDSS_REORDERING_ALG_COLAMD, CUDSS_REORDERING_ALG_BTF_COLAMD,
               CUDSS_REORDERING_ALG_NESTED_DISSECTION } cudssReorderingAlg_t;
typedef enum { CUDSS_MATCHING_ALG_AUTO = 0, CUDSS_MATCHING_ALG_NONE } cudssMatchingAlg_t;
typedef enum { CUDSS_PIVOT_AUTO = 0, CUDSS_PIVOT_GLOBAL_COL } cudssPivotType_t;
typedef enum { CUDSS_R_32I = 0, CUDSS_R_64F } cudssDataType_t;
typedef enum { CUDSS_CONFIG_REORDERING_ALG = 0, CUDSS_CONFIG_MATCHING_ALG, CUDSS_CONFIG_PIVOT_TYPE,
               CUDSS_CONFIG_PIVOT_THRESHOLD, CUDSS_CONFIG_UBATCH_SIZE } cudssConfigParam_t;
typedef enum { CUDSS_DATA_LU_NNZ = 0 } cudssDataParam_t;
typedef enum { CUDSS_PHASE_ANALYSIS = 1, CUDSS_PHASE_FACTORIZATION = 2, CUDSS_PHASE_REFACTORIZATION = 4,
               CUDSS_PHASE_SOLVE = 8 } cudssPhase_t;
cudssStatus_t cudssConfigSet(cudssConfig_t, cudssConfigParam_t, void *, size_t);
cudssStatus_t cudssDataGet(cudssHandle_t, cudssData_t, cudssDataParam_t, void *, size_t, size_t *);
cudssStatus_t cudssMatrixDestroy(cudssMatrix_t);
cudssStatus_t cudssDataDestroy(cudssHandle_t, cudssData_t);
cudssStatus_t cudssConfigDestroy(cudssConfig_t);
cudssStatus_t cudssDestroy(cudssHandle_t);
