/* fe_params.c -- FastEddy parameter-file reader (see fe_params.h for the contract).
 *
 * Storage is a flat array of entries searched linearly: a FastEddy file has a few
 * hundred keys at most and is read once, so a hash table buys nothing here.
 */
#include "fe_params.h"

#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define FE_MAX_ENTRIES 1024
#define FE_MAX_NAME 128
#define FE_MAX_VALUE 512

typedef struct {
  char name[FE_MAX_NAME];
  char value[FE_MAX_VALUE];
  int has_value;  /* 0 when the right-hand side was blank */
  int used;       /* set by any typed query */
} fe_entry;

static fe_entry g_entries[FE_MAX_ENTRIES];
static int g_count = 0;
static int g_errors = 0;
static char g_msg[512];

static void set_msg(const char *m, const char *name) {
  snprintf(g_msg, sizeof(g_msg), "%s%s%s", m, name ? ": " : "", name ? name : "");
}

void fe_params_reset(void) {
  g_count = 0;
  g_errors = 0;
  g_msg[0] = 0;
}

const char *fe_params_last_message(void) { return g_msg; }
int fe_params_error_count(void) { return g_errors; }

static char *trim(char *s) {
  char *e;
  while (*s && isspace((unsigned char)*s)) s++;
  e = s + strlen(s);
  while (e > s && isspace((unsigned char)e[-1])) e--;
  *e = 0;
  return s;
}

static fe_entry *find(const char *name) {
  int i;
  for (i = 0; i < g_count; i++)
    if (strcmp(g_entries[i].name, name) == 0) return &g_entries[i];
  return NULL;
}

static int parse_line(char *line) {
  char *hash, *eq, *name, *value;
  fe_entry *e;
  hash = strchr(line, '#');
  if (hash) *hash = 0;
  eq = strchr(line, '=');
  if (eq) {
    *eq = 0;
    value = trim(eq + 1);
  } else {
    value = (char *)"";
  }
  name = trim(line);
  if (name[0] == 0) return FE_PARAM_OK; /* blank or comment-only line */
  if (strlen(name) >= FE_MAX_NAME || strlen(value) >= FE_MAX_VALUE) {
    g_errors++;
    set_msg("parameter name or value too long", name);
    return FE_PARAM_ERR_SYNTAX;
  }
  if (find(name) != NULL) {
    g_errors++;
    set_msg("duplicate parameter", name);
    return FE_PARAM_ERR_DUPLICATE;
  }
  if (g_count >= FE_MAX_ENTRIES) {
    g_errors++;
    set_msg("too many parameters", name);
    return FE_PARAM_ERR_SYNTAX;
  }
  e = &g_entries[g_count++];
  strcpy(e->name, name);
  strcpy(e->value, value);
  e->has_value = value[0] != 0;
  e->used = 0;
  return FE_PARAM_OK;
}

int fe_params_read_text(const char *text) {
  int rc = FE_PARAM_OK;
  const char *p = text;
  char line[FE_MAX_NAME + FE_MAX_VALUE + 64];
  while (*p) {
    const char *nl = strchr(p, '\n');
    size_t n = nl ? (size_t)(nl - p) : strlen(p);
    if (n >= sizeof(line)) n = sizeof(line) - 1;
    memcpy(line, p, n);
    line[n] = 0;
    {
      int r = parse_line(line);
      if (r != FE_PARAM_OK) rc = r;
    }
    if (!nl) break;
    p = nl + 1;
  }
  return rc;
}

int fe_params_read_file(const char *path) {
  FILE *f = fopen(path, "r");
  char line[FE_MAX_NAME + FE_MAX_VALUE + 64];
  int rc = FE_PARAM_OK;
  if (!f) {
    g_errors++;
    set_msg("cannot open parameter file", path);
    return FE_PARAM_ERR_FILE;
  }
  while (fgets(line, sizeof(line), f) != NULL) {
    int r = parse_line(line);
    if (r != FE_PARAM_OK) rc = r;
  }
  fclose(f);
  return rc;
}

/* Shared lookup for typed queries: returns the entry, or NULL after applying the
 * absent-key rules (optional keeps *var, mandatory counts an error). */
static fe_entry *lookup_for_query(const char *name, int req, int *rc) {
  fe_entry *e = find(name);
  *rc = FE_PARAM_OK;
  if (e == NULL || !e->has_value) {
    if (e) e->used = 1;
    if (req == FE_PARAM_MANDATORY) {
      g_errors++;
      set_msg("mandatory parameter absent", name);
      *rc = FE_PARAM_ERR_ABSENT;
    } else if (req == FE_PARAM_OPTIONAL) {
      *rc = FE_PARAM_WARN_DEFAULTED;
    }
    return NULL;
  }
  e->used = 1;
  return e;
}

int fe_params_query_float(const char *name, float *var, float vmin, float vmax, int req) {
  int rc;
  float v;
  fe_entry *e = lookup_for_query(name, req, &rc);
  if (!e) return rc;
  if (sscanf(e->value, "%f", &v) != 1) {
    g_errors++;
    set_msg("not a float", name);
    return FE_PARAM_ERR_FLOAT;
  }
  if (v < vmin || v > vmax) {
    g_errors++;
    set_msg("float parameter outside its limits", name);
    return FE_PARAM_ERR_FLOAT;
  }
  *var = v;
  return FE_PARAM_OK;
}

int fe_params_query_int(const char *name, int *var, int vmin, int vmax, int req) {
  int rc;
  int v;
  fe_entry *e = lookup_for_query(name, req, &rc);
  if (!e) return rc;
  if (sscanf(e->value, "%d", &v) != 1) {
    g_errors++;
    set_msg("not an integer", name);
    return FE_PARAM_ERR_INTEGER;
  }
  if (v < vmin || v > vmax) {
    g_errors++;
    set_msg("integer parameter outside its limits", name);
    return FE_PARAM_ERR_INTEGER;
  }
  *var = v;
  return FE_PARAM_OK;
}

int fe_params_query_string(const char *name, const char **out, int req) {
  int rc;
  fe_entry *e = lookup_for_query(name, req, &rc);
  *out = e ? e->value : NULL;
  return rc;
}

int fe_params_report_unused(char *buf, int buflen) {
  int i, n = 0, off = 0;
  if (buf && buflen > 0) buf[0] = 0;
  for (i = 0; i < g_count; i++) {
    if (!g_entries[i].used) {
      n++;
      if (buf && off < buflen - 1) {
        int w = snprintf(buf + off, (size_t)(buflen - off), "%s%s", off ? " " : "", g_entries[i].name);
        if (w > 0) off += w;
      }
    }
  }
  return n;
}
