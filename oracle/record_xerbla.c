/*
 * record_xerbla.c -- test helper (checker infrastructure, never linked into the
 * product).  Defines a strong xerbla_ that records the routine name and info
 * code instead of printing them, so the tests can check the argument-error
 * behaviour of blas/level3_impl.h:61-78 (and of the product's dgemm_) exactly.
 * Loaded with RTLD_GLOBAL before the library under test, it interposes the weak
 * xerbla_ of blas/xerbla.cpp:18-20.
 */
#include <stddef.h>
#include <string.h>

static int g_last_info = 0;
static int g_calls = 0;
static char g_last_name[16];

void xerbla_(const char* name, int* info, size_t len) {
  g_last_info = info ? *info : -1;
  size_t n = len < sizeof(g_last_name) - 1 ? len : sizeof(g_last_name) - 1;
  memcpy(g_last_name, name, n);
  g_last_name[n] = 0;
  ++g_calls;
}

int record_xerbla_last_info(void) { return g_last_info; }
int record_xerbla_calls(void) { return g_calls; }
const char* record_xerbla_last_name(void) { return g_last_name; }
void record_xerbla_reset(void) {
  g_last_info = 0;
  g_calls = 0;
  g_last_name[0] = 0;
}
