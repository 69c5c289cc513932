// Minimal CBLAS prototypes (the names the reference's lib_dispatch.cpp calls),
// resolved at link time against the OpenBLAS shared library in the image.
#pragma once
extern "C" {
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
typedef CBLAS_ORDER CBLAS_LAYOUT;
void cblas_drot(int, double *, int, double *, int, double, double);
void cblas_srot(int, float *, int, float *, int, float, float);
void cblas_drotg(double *, double *, double *, double *);
void cblas_srotg(float *, float *, float *, float *);
double cblas_dnrm2(int, const double *, int);
float cblas_snrm2(int, const float *, int);
void cblas_dcopy(int, const double *, int, double *, int);
void cblas_scopy(int, const float *, int, float *, int);
double cblas_ddot(int, const double *, int, const double *, int);
float cblas_sdot(int, const float *, int, const float *, int);
void cblas_daxpy(int, double, const double *, int, double *, int);
void cblas_saxpy(int, float, const float *, int, float *, int);
void cblas_dscal(int, double, double *, int);
void cblas_sscal(int, float, float *, int);
void cblas_dgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int, int, double, const double *, int,
                 const double *, int, double, double *, int);
void cblas_sgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int, int, float, const float *, int,
                 const float *, int, float, float *, int);
void cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, double,
                 const double *, int, const double *, int, double, double *, int);
void cblas_sgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, float,
                 const float *, int, const float *, int, float, float *, int);
void cblas_dtpsv(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int, const double *,
                 double *, int);
void cblas_stpsv(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int, const float *,
                 float *, int);
}
