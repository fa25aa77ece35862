/*
 * NPY header reader/writer for oracle/shim/snpyio.h (oracle build only).
 * Format: NumPy's documented .npy layout, "\x93NUMPY", major/minor version,
 * little-endian header length (2 bytes for version 1, 4 for versions 2 and 3),
 * then a Python dict literal with 'descr', 'fortran_order' and 'shape',
 * space-padded and newline-terminated so the data starts on a 64-byte boundary.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>
#include "snpyio.h"

static const char magic[] = "\x93NUMPY";

/* find the value text following 'key': in the dict */
static const char * find_value(const char * dict, const char * key){
  char pattern[64];
  snprintf(pattern, sizeof(pattern), "'%s'", key);
  const char * p = strstr(dict, pattern);
  if(NULL == p) return NULL;
  p += strlen(pattern);
  while(*p && (isspace((unsigned char)*p) || ':' == *p)) p++;
  return p;
}

int snpyio_r_header(size_t * ndims, size_t ** shape, char ** dtype, bool * is_fortran_order, FILE * fp, size_t * header_size){
  unsigned char pre[10];
  if(8 != fread(pre, 1, 8, fp)) return 1;
  if(0 != memcmp(pre, magic, 6)) return 1;
  const int major = pre[6];
  size_t hlen = 0;
  size_t prelen = 0;
  if(1 == major){
    if(2 != fread(pre + 8, 1, 2, fp)) return 1;
    hlen = (size_t)pre[8] | ((size_t)pre[9] << 8);
    prelen = 10;
  }else if(2 == major || 3 == major){
    unsigned char l4[4];
    if(4 != fread(l4, 1, 4, fp)) return 1;
    hlen = (size_t)l4[0] | ((size_t)l4[1] << 8) | ((size_t)l4[2] << 16) | ((size_t)l4[3] << 24);
    prelen = 12;
  }else{
    return 1;
  }
  char * dict = calloc(hlen + 1, 1);
  if(hlen != fread(dict, 1, hlen, fp)){
    free(dict);
    return 1;
  }
  /* descr, kept with its quotes */
  const char * d = find_value(dict, "descr");
  if(NULL == d || '\'' != *d){
    free(dict);
    return 1;
  }
  const char * e = strchr(d + 1, '\'');
  if(NULL == e){
    free(dict);
    return 1;
  }
  const size_t dlen = (size_t)(e - d) + 1;
  *dtype = calloc(dlen + 1, 1);
  memcpy(*dtype, d, dlen);
  /* fortran_order */
  const char * f = find_value(dict, "fortran_order");
  if(NULL == f){
    free(dict);
    return 1;
  }
  *is_fortran_order = (0 == strncmp(f, "True", 4));
  /* shape tuple */
  const char * s = find_value(dict, "shape");
  if(NULL == s || '(' != *s){
    free(dict);
    return 1;
  }
  s++;
  size_t n = 0;
  size_t vals[32];
  while(*s && ')' != *s){
    while(*s && (isspace((unsigned char)*s) || ',' == *s)) s++;
    if(')' == *s) break;
    char * endp = NULL;
    const unsigned long long v = strtoull(s, &endp, 10);
    if(endp == s || n >= 32){
      free(dict);
      return 1;
    }
    vals[n++] = (size_t)v;
    s = endp;
  }
  *ndims = n;
  *shape = calloc(n > 0 ? n : 1, sizeof(size_t));
  for(size_t i = 0; i < n; i++){
    (*shape)[i] = vals[i];
  }
  *header_size = prelen + hlen;
  free(dict);
  return 0;
}

int snpyio_w_header(const size_t ndims, const size_t * shape, const char dtype[], const bool is_fortran_order, FILE * fp, size_t * header_size){
  char dict[1024];
  int len = snprintf(dict, sizeof(dict), "{'descr': %s, 'fortran_order': %s, 'shape': (", dtype, is_fortran_order ? "True" : "False");
  for(size_t i = 0; i < ndims; i++){
    len += snprintf(dict + len, sizeof(dict) - (size_t)len, "%zu%s", shape[i], (1 == ndims) ? "," : (i + 1 < ndims ? ", " : ""));
  }
  len += snprintf(dict + len, sizeof(dict) - (size_t)len, "), }");
  /* pad so that 10-byte preamble + dict + '\n' is a multiple of 64 */
  size_t total = 10 + (size_t)len + 1;
  const size_t padded = (total + 63) / 64 * 64;
  const size_t hlen = padded - 10;
  unsigned char pre[10];
  memcpy(pre, magic, 6);
  pre[6] = 1;
  pre[7] = 0;
  pre[8] = (unsigned char)(hlen & 0xff);
  pre[9] = (unsigned char)((hlen >> 8) & 0xff);
  if(10 != fwrite(pre, 1, 10, fp)) return 1;
  if((size_t)len != fwrite(dict, 1, (size_t)len, fp)) return 1;
  for(size_t i = (size_t)len; i + 1 < hlen; i++){
    fputc(' ', fp);
  }
  fputc('\n', fp);
  *header_size = padded;
  return 0;
}
