/* Declaration-only stand-in for SEPlib (the vendored copy needs flex, which is
 * absent here).  SEP I/O is host-side file handling, off the propagation
 * path; every function aborts if called (sep_stubs.cpp). */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
int putch(const char *name, const char *type, const void *val);
int auxputch(const char *name, const char *type, const void *val, const char *tag);
int hetch(const char *name, const char *type, void *val);
int auxpar(const char *name, const char *type, void *val, const char *tag);
long long sreed_big(const char *tag, void *buf, long long n);
long long srite_big(const char *tag, void *buf, long long n);
void initpar(int argc, char **argv);
#ifdef __cplusplus
}
#endif
