/* cudss.h -- compile-only stand-in for the cuDSS header, so that the
 * reference's 3D solver sources compile without the closed cuDSS library.
 *
 * TEST INFRASTRUCTURE ONLY.  It declares exactly the names that
 * src/FluidSim/FluidSolver3D.cu uses (its constructor, destructor and
 * pressureSolve), with argument lists written from those call sites.  The
 * definitions in cudss_stub.cpp do nothing: the constructor's cudssCreate
 * succeeds with a null handle, and every solve-side call reports
 * CUDSS_STATUS_NOT_SUPPORTED.  The fixture harness never calls pressureSolve. */
#ifndef FP_REFRUN_CUDSS_STUB_H
#define FP_REFRUN_CUDSS_STUB_H

#include <stdint.h>
#include <cuda_runtime.h>
#include <library_types.h>

typedef enum { CUDSS_STATUS_SUCCESS = 0, CUDSS_STATUS_NOT_SUPPORTED = 1 } cudssStatus_t;
typedef enum { CUDSS_MTYPE_SPD = 0 } cudssMatrixType_t;
typedef enum { CUDSS_MVIEW_UPPER = 0 } cudssMatrixViewType_t;
typedef enum { CUDSS_BASE_ZERO = 0 } cudssIndexBase_t;
typedef enum { CUDSS_LAYOUT_COL_MAJOR = 0 } cudssLayout_t;
typedef enum { CUDSS_PHASE_ANALYSIS = 1, CUDSS_PHASE_FACTORIZATION = 2, CUDSS_PHASE_SOLVE = 4 } cudssPhase_t;

typedef struct fpStubCudssHandle* cudssHandle_t;
typedef struct fpStubCudssConfig* cudssConfig_t;
typedef struct fpStubCudssData* cudssData_t;
typedef struct fpStubCudssMatrix* cudssMatrix_t;

cudssStatus_t cudssCreate(cudssHandle_t* handle);
cudssStatus_t cudssDestroy(cudssHandle_t handle);
cudssStatus_t cudssSetStream(cudssHandle_t handle, cudaStream_t stream);
cudssStatus_t cudssConfigCreate(cudssConfig_t* config);
cudssStatus_t cudssConfigDestroy(cudssConfig_t config);
cudssStatus_t cudssDataCreate(cudssHandle_t handle, cudssData_t* data);
cudssStatus_t cudssDataDestroy(cudssHandle_t handle, cudssData_t data);
cudssStatus_t cudssMatrixCreateCsr(cudssMatrix_t* m, int64_t nrows, int64_t ncols, int64_t nnz, void* row_start,
                                   void* row_end, void* col_ind, void* values, cudaDataType_t index_type,
                                   cudaDataType_t value_type, cudssMatrixType_t mtype, cudssMatrixViewType_t mview,
                                   cudssIndexBase_t base);
cudssStatus_t cudssMatrixCreateDn(cudssMatrix_t* m, int64_t nrows, int64_t ncols, int64_t ld, void* values,
                                  cudaDataType_t value_type, cudssLayout_t layout);
cudssStatus_t cudssMatrixDestroy(cudssMatrix_t m);
cudssStatus_t cudssExecute(cudssHandle_t handle, int phase, cudssConfig_t config, cudssData_t data,
                           cudssMatrix_t A, cudssMatrix_t x, cudssMatrix_t b);

#endif
