/*
 * Implementation of the argtable2 subset declared in argtable2.h (oracle
 * build only).  Accepts "-x v", "-xv", "--long=v" and "--long v"; flags are
 * counted.  Defaults match what the reference expects to read before it
 * checks `count` (src/util.c:138-150): 0 for numbers, "" for file names.
 */
#include "argtable2.h"
#include <stdlib.h>
#include <string.h>

static void *hdr_alloc(size_t sz, int kind, const char *s, const char *l, const char *g) {
  struct saru_arg_hdr *h = (struct saru_arg_hdr *)calloc(1, sz);
  if (!h) return NULL;
  h->kind = kind;
  h->shortopts = s;
  h->longopts = l;
  h->glossary = g;
  return h;
}

struct arg_int *arg_int0(const char *s, const char *l, const char *d, const char *g) {
  (void)d;
  struct arg_int *a = (struct arg_int *)hdr_alloc(sizeof(*a), SARU_ARG_INT, s, l, g);
  if (a) a->ival = (int *)calloc(1, sizeof(int));
  return a;
}

struct arg_dbl *arg_dbl0(const char *s, const char *l, const char *d, const char *g) {
  (void)d;
  struct arg_dbl *a = (struct arg_dbl *)hdr_alloc(sizeof(*a), SARU_ARG_DBL, s, l, g);
  if (a) a->dval = (double *)calloc(1, sizeof(double));
  return a;
}

struct arg_file *arg_file0(const char *s, const char *l, const char *d, const char *g) {
  (void)d;
  struct arg_file *a = (struct arg_file *)hdr_alloc(sizeof(*a), SARU_ARG_FILE, s, l, g);
  if (a) {
    a->filename = (const char **)calloc(1, sizeof(char *));
    if (a->filename) a->filename[0] = "";
  }
  return a;
}

struct arg_lit *arg_lit0(const char *s, const char *l, const char *g) {
  return (struct arg_lit *)hdr_alloc(sizeof(struct arg_lit), SARU_ARG_LIT, s, l, g);
}

struct arg_end *arg_end(int maxcount) {
  (void)maxcount;
  return (struct arg_end *)hdr_alloc(sizeof(struct arg_end), SARU_ARG_END, NULL, NULL, NULL);
}

int arg_nullcheck(void **argtable) {
  for (int i = 0;; i++) {
    struct saru_arg_hdr *h = (struct saru_arg_hdr *)argtable[i];
    if (!h) return 1;
    if (h->kind == SARU_ARG_END) return 0;
  }
}

static struct saru_arg_hdr *find_opt(void **argtable, const char *name, int is_long) {
  for (int i = 0;; i++) {
    struct saru_arg_hdr *h = (struct saru_arg_hdr *)argtable[i];
    if (h->kind == SARU_ARG_END) return NULL;
    if (is_long) {
      if (h->longopts && strcmp(h->longopts, name) == 0) return h;
    } else {
      if (h->shortopts && h->shortopts[0] == name[0]) return h;
    }
  }
}

static struct arg_end *find_end(void **argtable) {
  for (int i = 0;; i++) {
    struct saru_arg_hdr *h = (struct saru_arg_hdr *)argtable[i];
    if (h->kind == SARU_ARG_END) return (struct arg_end *)h;
  }
}

static int store(struct saru_arg_hdr *h, const char *val) {
  switch (h->kind) {
    case SARU_ARG_INT: {
      struct arg_int *a = (struct arg_int *)h;
      char *e;
      long v = strtol(val, &e, 0);
      if (*val == 0 || *e) return 1;
      a->ival[0] = (int)v;
      a->count++;
      return 0;
    }
    case SARU_ARG_DBL: {
      struct arg_dbl *a = (struct arg_dbl *)h;
      char *e;
      double v = strtod(val, &e);
      if (*val == 0 || *e) return 1;
      a->dval[0] = v;
      a->count++;
      return 0;
    }
    case SARU_ARG_FILE: {
      struct arg_file *a = (struct arg_file *)h;
      a->filename[0] = val;
      a->count++;
      return 0;
    }
    default:
      return 1;
  }
}

int arg_parse(int argc, char **argv, void **argtable) {
  struct arg_end *end = find_end(argtable);
  int errors = 0;
  for (int i = 1; i < argc; i++) {
    const char *a = argv[i];
    struct saru_arg_hdr *h = NULL;
    const char *inline_val = NULL;
    if (a[0] == '-' && a[1] == '-') {
      char name[128];
      const char *eq = strchr(a + 2, '=');
      size_t n = eq ? (size_t)(eq - (a + 2)) : strlen(a + 2);
      if (n >= sizeof(name)) n = sizeof(name) - 1;
      memcpy(name, a + 2, n);
      name[n] = 0;
      h = find_opt(argtable, name, 1);
      if (eq) inline_val = eq + 1;
    } else if (a[0] == '-' && a[1]) {
      h = find_opt(argtable, a + 1, 0);
      if (a[2]) inline_val = a + 2;
    }
    if (!h) {
      snprintf(end->message, sizeof(end->message), "unexpected argument \"%s\"", a);
      errors++;
      continue;
    }
    if (h->kind == SARU_ARG_LIT) {
      ((struct arg_lit *)h)->count++;
      continue;
    }
    const char *val = inline_val;
    if (!val) {
      if (i + 1 >= argc) {
        snprintf(end->message, sizeof(end->message), "option \"%s\" needs a value", a);
        errors++;
        continue;
      }
      val = argv[++i];
    }
    if (store(h, val)) {
      snprintf(end->message, sizeof(end->message), "invalid value \"%s\"", val);
      errors++;
    }
  }
  end->count = errors;
  return errors;
}

void arg_print_syntax(FILE *fp, void **argtable, const char *suffix) {
  for (int i = 0;; i++) {
    struct saru_arg_hdr *h = (struct saru_arg_hdr *)argtable[i];
    if (h->kind == SARU_ARG_END) break;
    if (h->shortopts) fprintf(fp, " [-%s]", h->shortopts);
  }
  fputs(suffix, fp);
}

void arg_print_glossary(FILE *fp, void **argtable, const char *format) {
  for (int i = 0;; i++) {
    struct saru_arg_hdr *h = (struct saru_arg_hdr *)argtable[i];
    if (h->kind == SARU_ARG_END) break;
    fprintf(fp, format, h->longopts ? h->longopts : "", h->glossary ? h->glossary : "");
  }
}

void arg_print_errors(FILE *fp, struct arg_end *end, const char *progname) {
  fprintf(fp, "%s: %s\n", progname, end->message);
}

void arg_freetable(void **argtable, size_t n) {
  for (size_t i = 0; i < n; i++) {
    struct saru_arg_hdr *h = (struct saru_arg_hdr *)argtable[i];
    if (!h) continue;
    switch (h->kind) {
      case SARU_ARG_INT: free(((struct arg_int *)h)->ival); break;
      case SARU_ARG_DBL: free(((struct arg_dbl *)h)->dval); break;
      case SARU_ARG_FILE: free((void *)((struct arg_file *)h)->filename); break;
      default: break;
    }
    free(h);
    argtable[i] = NULL;
  }
}
