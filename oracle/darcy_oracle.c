/*
 * Darcy pressure solver for the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 * (Filled in with the Darcy restatement; for now the section is parsed so
 * that fluid files load.)
 */
#include "sph_oracle.h"
#include "oracle_internal.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct orc_darcy { int unused; };

int orc_darcy_load(orc_state *s, const unsigned char **cur, const unsigned char *end)
{
    (void)s; (void)cur; (void)end;
    return ORC_ERR_UNSUPPORTED;
}
int orc_darcy_step(orc_state *s)
{
    orc_set_error(s, ORC_ERR_UNSUPPORTED, "Darcy solver not built");
    return s->err;
}
int orc_darcy_write(orc_state *s, void *fh) { (void)s; (void)fh; return 0; }
void orc_darcy_free(orc_state *s) { free(s->darcy); s->darcy = NULL; }
int64_t orc_darcy_get(orc_state *s, const char *name, void *dst, size_t bytes)
{
    (void)s; (void)name; (void)dst; (void)bytes;
    return -1;
}
