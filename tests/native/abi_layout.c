/* Compiled as plain C99 against include/evp1d.h and linked with the library:
 * prints the size and field offsets of the public structs, then makes a few
 * host-only calls (no GPU needed).  Test code only. */
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include "evp1d.h"

#define F(T, m) printf("%s.%s %zu\n", #T, #m, offsetof(T, m))

int main(void) {
  printf("evp1d_params %zu\n", sizeof(evp1d_params));
  F(evp1d_params, arlx1i); F(evp1d_params, deltaminEVP); F(evp1d_params, rhow);
  printf("evp1d_fields %zu\n", sizeof(evp1d_fields));
  F(evp1d_fields, skipT); F(evp1d_fields, stress); F(evp1d_fields, strength);
  F(evp1d_fields, Tbu); F(evp1d_fields, uvel_init); F(evp1d_fields, uvel);
  F(evp1d_fields, Cb); F(evp1d_fields, str);
  printf("evp1d_grads %zu\n", sizeof(evp1d_grads));
  F(evp1d_grads, strength); F(evp1d_grads, stress); F(evp1d_grads, vvel_init);
  printf("evp1d_dyn_fields %zu\n", sizeof(evp1d_dyn_fields));
  F(evp1d_dyn_fields, stress); F(evp1d_dyn_fields, strength); F(evp1d_dyn_fields, Tbu);
  F(evp1d_dyn_fields, uvel); F(evp1d_dyn_fields, iceumask);

  evp1d_params p;
  evp1d_set_evp_parameters(&p, 120);
  printf("brlx %.1f\n", p.brlx);
  /* a NULL handle is refused with a message, not a crash */
  const int rc = evp1d_run(NULL, 120, NULL);
  printf("run_null %d,%d\n", rc, (int)(strlen(evp1d_last_error()) > 0));
  printf("version %d\n", (int)(strlen(evp1d_version()) > 0));
  return 0;
}
