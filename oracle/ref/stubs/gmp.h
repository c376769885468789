#ifndef ORACLE_STUB_GMP_H
#define ORACLE_STUB_GMP_H
typedef struct
{
  int a, s;
  void *d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
#endif
