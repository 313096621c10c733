"""The MEX gateway (mex/ufvm_mex.c) against the C-ABI header: there is no MATLAB here, so the
gateway is compiled with gcc -fsyntax-only against stand-in declarations of the MEX and
mxGPUArray functions it calls (names and signatures as MATLAB's external-interface documents
describe them), with and without its gpuArray commands. A change of include/ufvm.h that the
gateway does not follow fails here."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MEX_H = r"""
#pragma once
#include <stddef.h>
#include <stdbool.h>
#include <stdint.h>
typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS, mxDOUBLE_CLASS, mxINT32_CLASS, mxUINT64_CLASS } mxClassID;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;
typedef bool mxLogical;
double mxGetScalar(const mxArray*);
mxArray* mxCreateDoubleScalar(double);
mxArray* mxCreateDoubleMatrix(mwSize, mwSize, mxComplexity);
mxArray* mxCreateNumericMatrix(mwSize, mwSize, mxClassID, mxComplexity);
mxArray* mxCreateLogicalScalar(mxLogical);
mxArray* mxCreateString(const char*);
mxArray* mxCreateStructMatrix(mwSize, mwSize, int, const char**);
double* mxGetDoubles(const mxArray*);
int32_t* mxGetInt32s(const mxArray*);
uint64_t* mxGetUint64s(const mxArray*);
int mxGetString(const mxArray*, char*, mwSize);
mwSize mxGetNumberOfElements(const mxArray*);
mxArray* mxGetField(const mxArray*, mwIndex, const char*);
void mxSetField(mxArray*, mwIndex, const char*, mxArray*);
bool mxIsEmpty(const mxArray*);
bool mxIsUint64(const mxArray*);
bool mxIsStruct(const mxArray*);
bool mxIsInt32(const mxArray*);
bool mxIsDouble(const mxArray*);
bool mxIsComplex(const mxArray*);
bool mxIsChar(const mxArray*);
int mexAtExit(void (*)(void));
void mexErrMsgIdAndTxt(const char*, const char*, ...);
void mexFunction(int, mxArray* [], int, const mxArray* []);
"""

GPU_H = r"""
#pragma once
#include "mex.h"
typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_INITIALIZE_VALUES, MX_GPU_DO_NOT_INITIALIZE } mxGPUInitialize;
int mxInitGPU(void);
const mxGPUArray* mxGPUCreateFromMxArray(const mxArray*);
mxGPUArray* mxGPUCopyFromMxArray(const mxArray*);
void* mxGPUGetData(mxGPUArray*);
const void* mxGPUGetDataReadOnly(const mxGPUArray*);
mwSize mxGPUGetNumberOfElements(const mxGPUArray*);
mxClassID mxGPUGetClassID(const mxGPUArray*);
mxGPUArray* mxGPUCreateGPUArray(mwSize, const mwSize*, mxClassID, mxComplexity, mxGPUInitialize);
mxArray* mxGPUCreateMxArrayOnGPU(const mxGPUArray*);
void mxGPUDestroyGPUArray(const mxGPUArray*);
"""


@pytest.mark.parametrize("gpu", [False, True], ids=["case_and_service", "with_gpuarray"])
def test_mex_gateway_compiles_against_the_header(tmp_path, gpu):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    (tmp_path / "gpu").mkdir()
    (tmp_path / "mex.h").write_text(MEX_H)
    (tmp_path / "gpu" / "mxGPUArray.h").write_text(GPU_H)
    cmd = [gcc, "-std=c11", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I", str(tmp_path),
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "mex", "ufvm_mex.c")]
    if gpu:
        cmd.insert(1, "-DUFVM_MEX_GPU")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
