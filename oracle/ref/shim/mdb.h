/*
 * TEST INFRASTRUCTURE (oracle/ref): a minimal stand-in for the SDDS toolkit
 * headers (mdb.h, SDDS.h, namelist.h, table.h, constants.h, matlib.h, ...)
 * that elegant's sources include but that are not shipped with elegant.
 * Written for this project from the way elegant's tracking sources use these
 * names.  Numerical helpers (sqr, ipow, SIGN, KahanPlus, compute_average, the
 * physical constants) restate the SDDS toolkit's published definitions and
 * use the same constants as the CUDA library (elegant_b200/csrc/
 * trk_constants.h), so that a comparison tests elegant's algorithms, not the
 * constants.  Everything else (file I/O, namelists, RPN, matrices) is
 * declared so the sources compile; the oracle never reaches it, and
 * oracle/ref/stubs.c aborts if it ever does.
 */
#ifndef ORACLE_REF_SHIM_MDB_H
#define ORACLE_REF_SHIM_MDB_H

#include <ctype.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------- constants */
#define PI 3.141592653589793238462643
#define PIx2 6.283185307179586476925287
#define PIo2 1.570796326794896619231322
#define SQRT2 1.414213562373095048801689
#define c_mks 2.99792458e8
#define c_cgs 2.99792458e10
#define e_mks 1.602176634e-19
#define me_mks 9.1093837015e-31
#define me_mev 0.51099895000
#define mp_mks 1.67262192369e-27
#define mp_mev 938.27208816
#define re_mks 2.8179403262e-15
#define mu_o (4 * PI * 1e-7)
#define epsilon_o (1 / (mu_o * c_mks * c_mks))
#define hbar_mks 1.054571817e-34
#define k_boltzmann_mks 1.380649e-23
#define SVN_VERSION "shim"

/* -------------------------------------------------------- small helpers */
#define sqr(x) ((x) * (x))
#define FABS(x) fabs(x)
#define INTERPOLATE(y1, y2, x1, x2, x) ((y1) + ((y2) - (y1)) * ((x) - (x1)) / ((x2) - (x1)))
#define SIGN(x) ((x) < 0 ? -1 : 1)
#ifndef MIN
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#endif
#define SWAP_DOUBLE(a, b)                                                                                        \
  do {                                                                                                           \
    double swap_tmp_ = (a);                                                                                      \
    (a) = (b);                                                                                                   \
    (b) = swap_tmp_;                                                                                             \
  } while (0)
#define SWAP_LONG(a, b)                                                                                          \
  do {                                                                                                           \
    long swap_tmp_ = (a);                                                                                        \
    (a) = (b);                                                                                                   \
    (b) = swap_tmp_;                                                                                             \
  } while (0)
#define SWAP_PTR(a, b)                                                                                           \
  do {                                                                                                           \
    void *swap_tmp_ = (a);                                                                                       \
    (a) = (b);                                                                                                   \
    (b) = swap_tmp_;                                                                                             \
  } while (0)

double ipow(double x, long p);
double ipow1(double x);
double ipow7(double x);
int double_cmpasc(const void *a, const void *b);
double ipow2(double x);
double ipow3(double x);
double ipow4(double x);
double ipow5(double x);
double ipow6(double x);
double pow2(double x);
double pow3(double x);
double pow4(double x);
double pow5(double x);
double dfactorial(long n);
double KahanPlus(double sum, double b, double *error);
long compute_average(double *value, double *x, long n);

void *tmalloc(uint64_t size);
void *trealloc(void *ptr, uint64_t size);
int tfree(void *ptr);
void **czarray_2d(uint64_t size, uint64_t n1, uint64_t n2);
int free_czarray_2d(void **array, uint64_t n1, uint64_t n2);
void **zarray_2d(uint64_t size, uint64_t n1, uint64_t n2);
int free_zarray_2d(void **array, uint64_t n1, uint64_t n2);
char *cp_str(char **s, char *t);
void bomb(char *error, char *usage);
void log_entry(const char *routine);
void log_exit(const char *routine);
void push_log();
void pop_log();

/* ---------------------------------------------- opaque SDDS toolkit types */
typedef struct {
  int shim_unused;
} SDDS_DATASET;
typedef SDDS_DATASET SDDS_TABLE;
typedef struct {
  char *name;
} SDDS_DEFINITION;
typedef struct {
  int shim_unused;
} NAMELIST_TEXT;
typedef struct {
  int shim_unused;
} htab;
typedef struct {
  double **a;
  long n, m;
} MATRIX;
typedef struct {
  double *c1, *c2, *s1, *s2;
  long n_data, flags;
  char *xlab, *ylab, *topline, *title;
} TABLE;

#define SDDS_BINARY 1
#define SDDS_ASCII 2
#define SDDS_DOUBLE 1
#define SDDS_FLOAT 2
#define SDDS_LONG64 3
#define SDDS_ULONG64 4
#define SDDS_LONG 5
#define SDDS_ULONG 6
#define SDDS_SHORT 7
#define SDDS_USHORT 8
#define SDDS_STRING 9
#define SDDS_CHARACTER 10
#define SDDS_LONGDOUBLE 11
#define SDDS_ANY_NUMERIC_TYPE 99
#define SDDS_ANY_FLOATING_TYPE 98
#define SDDS_ANY_INTEGER_TYPE 97
#define SDDS_CHECK_OK 0
#define SDDS_CHECK_NONEXISTENT 1
#define SDDS_CHECK_WRONGTYPE 2
#define SDDS_CHECK_WRONGUNITS 3
#define SDDS_VERBOSE_PrintErrors 1
#define SDDS_EXIT_PrintErrors 2
#define SDDS_SET_BY_INDEX 1
#define SDDS_SET_BY_NAME 2
#define SDDS_PASS_BY_VALUE 1
#define SDDS_PASS_BY_REFERENCE 2
#define SDDS_PASS_BY_STRING 4
#define SDDS_ROW_MAJOR_DATA 1
#define SDDS_COLUMN_MAJOR_DATA 2
#define INVERSE_FFT 1
#define FLUSH_TABLE 1
#define SDDS_IDENTIFIER_ERRORS 0
#define SDDS_BY_NAME 1
#define SDDS_BY_INDEX 2

/* unprototyped: never called on the oracle's paths (stubs.c aborts) */
long SDDS_CheckColumn();
long SDDS_CheckParameter();
long SDDS_RowCount();
long SDDS_ReadPage();
long SDDS_Terminate();
long SDDS_InitializeInputFromSearchPath();
long SDDS_InitializeInput();
long SDDS_InitializeOutput();
long SDDS_WriteLayout();
long SDDS_WritePage();
long SDDS_StartPage();
long SDDS_SetRowValues();
long SDDS_SetParameters();
long SDDS_SetColumn();
long SDDS_DefineColumn();
long SDDS_DefineParameter();
long SDDS_DefineSimpleColumn();
long SDDS_DefineSimpleParameter();
long SDDS_GetColumnIndex();
long SDDS_GetParameterIndex();
long SDDS_CopyString();
long SDDS_GetColumnInformation();
long SDDS_SetError();
long SDDS_Bomb();
long SDDS_PrintErrors();
long SDDS_DoFSync();
long SDDS_SaveLayout();
long SDDS_CountRowsOfInterest();
long SDDS_GetParameterAsDouble();
long SDDS_GetParameterAsLong();
double *SDDS_GetColumnInDoubles();
void *SDDS_GetColumn();
void *SDDS_GetParameter();
void *SDDS_Malloc();
void *SDDS_Realloc();
void *SDDS_Calloc();
char **SDDS_GetColumnNames();
long SDDS_UpdatePage();
long SDDS_SetColumnFromDoubles();
long SDDS_SetColumnFromLongs();
long SDDS_ClearErrors();
long SDDS_NumberOfErrors();
long SDDS_GetParameterByIndex();
long SDDS_ChangeColumnInformation();
long SDDS_ChangeParameterInformation();
long SDDS_LengthenTable();
long SDDS_DisconnectFile();
long SDDS_ReconnectFile();
long SDDS_GetNamedColumnType();
long SDDS_FreeStringArray();
long SDDS_SetNoRowCounts();
long SDDS_ForceInactive();
long SDDS_IsActive();
long SDDS_TransferAllParameterDefinitions();
long SDDS_TransferColumnDefinition();
long SDDS_TransferParameterDefinition();
long SDDS_CopyPage();
long SDDS_CopyParameters();
long match_string();
/* match_string modes (values of this shim: match_string is not on the tracking path) */
#define DCL_STYLE_MATCH 0x0001
#define UNIQUE_MATCH 0x0002
#define CASE_SENSITIVE 0x0004
#define MATCH_WHOLE_STRING 0x0008
#define EXACT_MATCH (CASE_SENSITIVE | MATCH_WHOLE_STRING)
long str_in();
long fexists();
long get_long();
long get_double();
char *compose_filename();
long SavitzyGolaySmooth();
long find_min_max();
long realFFT2();
double zeroNewton();
double zeroInterp();
long simplexMin();
long rpn_clear();
double rpn();
long rpn_store();
long rpn_create_mem();
long log_and();
long log_or();
double gauss_rn_lim();
double gauss_rn();
double random_1();
double random_2();
double random_3();
double random_4();
long m_alloc();
long m_free();
long m_trans();
long m_mult();
long m_zero();
long m_subtract();
long m_scmul();
long m_invert();
long m_copy();
long m_add();
long m_show();
long m_check();
long m_identity();
long m_bomb();
long m_det();
double interp();
long index_min_max();
double getTimeInSecs();
FILE *fopen_e();
long fill_double_array();
long compute_percentiles();
long bitsSet();
long binaryArraySearch();
long SavitzkyGolaySmooth();
int32_t *SDDS_GetColumnInLong();

#endif
