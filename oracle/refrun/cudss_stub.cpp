// cudss_stub.cpp -- do-nothing definitions for the compile-only cuDSS header
// (cudss.h beside this file).  TEST INFRASTRUCTURE ONLY: lets the reference's
// FluidSolver3D be constructed and destroyed; nothing here solves anything.
#include "cudss.h"

cudssStatus_t cudssCreate(cudssHandle_t* handle) { *handle = nullptr; return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssDestroy(cudssHandle_t) { return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssSetStream(cudssHandle_t, cudaStream_t) { return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssConfigCreate(cudssConfig_t* config) { *config = nullptr; return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssConfigDestroy(cudssConfig_t) { return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssDataCreate(cudssHandle_t, cudssData_t* data) { *data = nullptr; return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssDataDestroy(cudssHandle_t, cudssData_t) { return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssMatrixCreateCsr(cudssMatrix_t* m, int64_t, int64_t, int64_t, void*, void*, void*, void*,
                                   cudaDataType_t, cudaDataType_t, cudssMatrixType_t, cudssMatrixViewType_t,
                                   cudssIndexBase_t) {
    *m = nullptr;
    return CUDSS_STATUS_NOT_SUPPORTED;
}
cudssStatus_t cudssMatrixCreateDn(cudssMatrix_t* m, int64_t, int64_t, int64_t, void*, cudaDataType_t, cudssLayout_t) {
    *m = nullptr;
    return CUDSS_STATUS_NOT_SUPPORTED;
}
cudssStatus_t cudssMatrixDestroy(cudssMatrix_t) { return CUDSS_STATUS_SUCCESS; }
cudssStatus_t cudssExecute(cudssHandle_t, int, cudssConfig_t, cudssData_t, cudssMatrix_t, cudssMatrix_t,
                           cudssMatrix_t) {
    return CUDSS_STATUS_NOT_SUPPORTED;
}
