/*
 * Minimal command-line parser exposing the subset of the argtable2 interface
 * that the reference's src/util.c:59-290 uses (arg_int0, arg_dbl0, arg_file0,
 * arg_lit0, arg_end, arg_nullcheck, arg_parse, arg_print_*, arg_freetable).
 * libargtable2 is not installed in this image; this shim exists only so the
 * reference's host C can be linked into oracle/_ref test binaries.  Field
 * names (count, ival, dval, filename) follow the argtable2 interface because
 * the reference reads them directly.
 */
#ifndef SARU_REF_SHIM_ARGTABLE2_H
#define SARU_REF_SHIM_ARGTABLE2_H
#include <stdio.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

enum saru_arg_kind { SARU_ARG_INT, SARU_ARG_DBL, SARU_ARG_FILE, SARU_ARG_LIT, SARU_ARG_END };

struct saru_arg_hdr {
  int kind;
  const char *shortopts;
  const char *longopts;
  const char *glossary;
};

struct arg_int { struct saru_arg_hdr hdr; int count; int *ival; };
struct arg_dbl { struct saru_arg_hdr hdr; int count; double *dval; };
struct arg_file { struct saru_arg_hdr hdr; int count; const char **filename; };
struct arg_lit { struct saru_arg_hdr hdr; int count; };
struct arg_end { struct saru_arg_hdr hdr; int count; char message[256]; };

struct arg_int *arg_int0(const char *s, const char *l, const char *d, const char *g);
struct arg_dbl *arg_dbl0(const char *s, const char *l, const char *d, const char *g);
struct arg_file *arg_file0(const char *s, const char *l, const char *d, const char *g);
struct arg_lit *arg_lit0(const char *s, const char *l, const char *g);
struct arg_end *arg_end(int maxcount);
int arg_nullcheck(void **argtable);
int arg_parse(int argc, char **argv, void **argtable);
void arg_print_syntax(FILE *fp, void **argtable, const char *suffix);
void arg_print_glossary(FILE *fp, void **argtable, const char *format);
void arg_print_errors(FILE *fp, struct arg_end *end, const char *progname);
void arg_freetable(void **argtable, size_t n);

#ifdef __cplusplus
}
#endif
#endif
