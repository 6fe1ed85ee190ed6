/*
 * input.c -- the input.dat keyword format.
 *
 * The format is a list of "name, value" lines. Its accepted inputs are defined by the state machine of
 * inputInit (input.c:7-95 of the reference), which this file follows so that every input.dat the
 * reference accepts is read identically:
 *   - ' ' and '\r' are dropped everywhere (so "a b" reads as "ab");
 *   - ',' ends the name and starts the value;
 *   - '#' ends the value and switches recording off without resetting the column; recording resumes
 *     (into the value) only at the next ',', so a comment normally drops its own entry;
 *   - '\n' closes an entry that has a value, or a name-only entry with at least one character.
 * An entry is only counted at a '\n'. Lookups return the LAST entry of a repeated name
 * (inputGetValue, input.c:122-143). Differences: names/values longer than 49 characters and more than
 * 100 entries are rejected with CSU_ERR_INPUT (the reference overflows its buffers), and a missing
 * keyword is reported to the caller instead of exit(0).
 */
#include <string.h>
#include "case.h"

int csu_keywords_parse(const char* text, size_t len, csu_keywords* kw)
{
    int in_name = 1, in_value = 0, ii = 0, jj = 0;
    memset(kw, 0, sizeof(*kw));
    for (size_t pos = 0; pos < len; pos++) {
        char c = text[pos];
        if (c == ' ' || c == '\r') continue;
        if (ii >= CSU_KW_MAX && (c != '\n' || in_value || (in_name && jj > 0))) {
            csu_set_error("input.dat: more than %d entries", CSU_KW_MAX);
            return CSU_ERR_INPUT;
        }
        if (c == ',') {
            in_name = 0;
            in_value = 1;
            kw->name[ii][jj] = '\0';
            jj = 0;
        } else if (c == '#') {
            in_name = 0;
            in_value = 0;
            kw->value[ii][jj] = '\0';
        } else if (c == '\n') {
            if (in_value) {
                in_name = 1;
                in_value = 0;
                kw->value[ii][jj] = '\0';
                ii++;
                jj = 0;
            }
            if (in_name && jj > 0) {
                kw->name[ii][jj] = '\0';
                ii++;
                jj = 0;
            }
        } else if (in_name || in_value) {
            if (jj >= CSU_KW_LEN - 1) {
                csu_set_error("input.dat: entry %d longer than %d characters", ii, CSU_KW_LEN - 1);
                return CSU_ERR_INPUT;
            }
            if (in_name) kw->name[ii][jj++] = c;
            else kw->value[ii][jj++] = c;
        }
    }
    kw->n = ii;
    return CSU_OK;
}

int csu_keywords_has(const csu_keywords* kw, const char* name)
{
    for (int i = 0; i < kw->n; i++)
        if (strcmp(name, kw->name[i]) == 0) return 1;
    return 0;
}

const char* csu_keywords_get(const csu_keywords* kw, const char* name)
{
    const char* s = NULL;
    for (int i = 0; i < kw->n; i++)
        if (strcmp(name, kw->name[i]) == 0) s = kw->value[i];
    return s;
}
