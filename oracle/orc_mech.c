/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle.h; parity unpinned).
 *
 * Restatement of the reference mechanism and thermo readers, including the
 * Fortran list-directed input rules they rely on:
 *   - a READ(*) of a character item takes the first value of the next record
 *     that holds one: blank records are skipped, an undelimited value ends at a
 *     blank, comma or slash, a quoted value runs to the closing quote;
 *   - BACKSPACE steps back over the last record that READ consumed;
 *   - reals may omit the exponent letter ("4.8749+04").
 * Reference: package_library/src/chemical_properties_class.f90:117-181 (set
 * properties), :222-287 (reaction count), :289-451 (reaction properties),
 * :453-635 (reaction string parser), :637-655 (species lookup), :685-768
 * (species readers); thermophysical_properties_class.f90:137-210 (set
 * properties), :1226-1311 (NASA-7 tokenizer), :1313-1341 (molar mass).
 */
#include "oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define R_GASE_J 8.31446261815324
#define R_GASE_CAL 1.98720425864083

/* ------------------------------------------------------------------ file */
typedef struct {
    char **lines;
    int n;
    int pos; /* index of next record */
} recfile;

static int rf_open(recfile *f, const char *path) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return -1;
    fseek(fp, 0, SEEK_END);
    long sz = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)sz + 1);
    if (!buf) { fclose(fp); return -1; }
    size_t got = fread(buf, 1, (size_t)sz, fp);
    fclose(fp);
    buf[got] = 0;
    int cap = 64;
    f->lines = (char **)malloc(sizeof(char *) * cap);
    f->n = 0;
    f->pos = 0;
    char *p = buf;
    while (*p || p == buf) {
        char *e = strchr(p, '\n');
        size_t len = e ? (size_t)(e - p) : strlen(p);
        if (len > 0 && p[len - 1] == '\r') len--;
        if (f->n == cap) { cap *= 2; f->lines = (char **)realloc(f->lines, sizeof(char *) * cap); }
        char *l = (char *)malloc(len + 1);
        memcpy(l, p, len);
        l[len] = 0;
        f->lines[f->n++] = l;
        if (!e) break;
        p = e + 1;
        if (!*p) break;
    }
    free(buf);
    return 0;
}

static void rf_close(recfile *f) {
    for (int i = 0; i < f->n; i++) free(f->lines[i]);
    free(f->lines);
    f->lines = NULL;
    f->n = 0;
}

static int is_blank(char c) { return c == ' ' || c == '\t'; }

/* One list-directed value scanner positioned inside a record. */
typedef struct {
    recfile *f;
    const char *p; /* current char in record, NULL = need next record */
    int first_rec; /* index of record where this READ started */
} ldscan;

/* Fetch the next value token (may cross records).  Returns 1 and fills tok,
 * 0 on end of file, -1 on a slash terminator. */
static int ld_next(ldscan *s, char *tok, size_t cap) {
    for (;;) {
        if (!s->p) {
            if (s->f->pos >= s->f->n) return 0;
            s->p = s->f->lines[s->f->pos++];
        }
        while (*s->p && (is_blank(*s->p) || *s->p == ',')) {
            /* a comma between values separates; a leading comma would be a
             * null value, which the reference files never contain */
            s->p++;
        }
        if (!*s->p) { s->p = NULL; continue; }
        if (*s->p == '/') return -1;
        size_t k = 0;
        if (*s->p == '\'' || *s->p == '"') {
            char q = *s->p++;
            while (*s->p) {
                if (*s->p == q) {
                    if (s->p[1] == q) { if (k + 1 < cap) tok[k++] = q; s->p += 2; continue; }
                    s->p++;
                    break;
                }
                if (k + 1 < cap) tok[k++] = *s->p;
                s->p++;
            }
        } else {
            while (*s->p && !is_blank(*s->p) && *s->p != ',' && *s->p != '/') {
                if (k + 1 < cap) tok[k++] = *s->p;
                s->p++;
            }
        }
        tok[k] = 0;
        return 1;
    }
}

/* READ(u,*) string : returns 1 ok, 0 EOF */
static int ld_read_string(recfile *f, char *out, size_t cap) {
    ldscan s = {f, NULL, f->pos};
    int r = ld_next(&s, out, cap);
    return r == 1;
}

static void rf_backspace(recfile *f) { if (f->pos > 0) f->pos--; }

/* Fortran real literal (list-directed) -> double.  Returns 0 on success. */
static int fortran_real(const char *tok, double *out) {
    char buf[128];
    size_t k = 0;
    const char *p = tok;
    while (is_blank(*p)) p++;
    if (*p == '+' || *p == '-') buf[k++] = *p++;
    int nd = 0;
    while (isdigit((unsigned char)*p) || *p == '.') { if (k < 100) buf[k++] = *p; if (*p != '.') nd++; p++; }
    if (nd == 0) return -1;
    if (*p == 'E' || *p == 'e' || *p == 'D' || *p == 'd' || *p == 'Q' || *p == 'q') {
        buf[k++] = 'E';
        p++;
        if (*p == '+' || *p == '-') buf[k++] = *p++;
        if (!isdigit((unsigned char)*p)) return -1;
        while (isdigit((unsigned char)*p)) { if (k < 120) buf[k++] = *p; p++; }
    } else if (*p == '+' || *p == '-') {
        buf[k++] = 'E';
        buf[k++] = *p++;
        if (!isdigit((unsigned char)*p)) return -1;
        while (isdigit((unsigned char)*p)) { if (k < 120) buf[k++] = *p; p++; }
    }
    while (is_blank(*p)) p++;
    if (*p) return -1;
    buf[k] = 0;
    *out = strtod(buf, NULL);
    return 0;
}

/* Trimmed (trailing blanks) Fortran string equality. */
static int fstr_eq(const char *a, const char *b) {
    size_t la = strlen(a), lb = strlen(b);
    while (la > 0 && a[la - 1] == ' ') la--;
    while (lb > 0 && b[lb - 1] == ' ') lb--;
    return la == lb && strncmp(a, b, la) == 0;
}

/* ---------------------------------------------------------- species */
static int specie_index(const orc_mech *m, const char *name) {
    /* get_chemical_specie_index: 1-based over species + "M" (n+1) */
    for (int i = 0; i <= m->n_species; i++)
        if (fstr_eq(name, m->species_names[i])) return i + 1;
    return 0;
}

/* read_chemical_species_number / names: character-by-character tokenizer
 * of the records after SPECIES, stopping at END. */
static int read_species(recfile *f, orc_mech *m) {
    char tok[256];
    f->pos = 0;
    for (;;) {
        if (!ld_read_string(f, tok, sizeof tok)) return -1;
        if (fstr_eq(tok, "SPECIES")) break;
    }
    /* non-advancing single-character reads; end of record pads with blank */
    int rec = f->pos;
    const char *p = rec < f->n ? f->lines[rec] : NULL;
    int n = 0;
    for (;;) {
        char s[160];
        memset(s, ' ', sizeof s);
        int i = 2; /* 0-based position of string(3:3) */
        char letter = 'x';
        while (letter != ' ' || s[i - 2] == ' ') {
            if (!p) return -1;
            if (*p) {
                letter = *p++;
                if (letter == '\t') letter = '\t';
            } else {
                letter = ' ';
                rec++;
                p = rec < f->n ? f->lines[rec] : NULL;
            }
            if (i < (int)sizeof s - 1) s[i] = letter;
            i++;
            if (i >= (int)sizeof s - 1) return -1;
        }
        s[i] = 0;
        /* trim(adjustl(string)) */
        char *a = s;
        while (*a == ' ') a++;
        size_t L = strlen(a);
        while (L > 0 && (a[L - 1] == ' ')) L--;
        a[L] = 0;
        if (fstr_eq(a, "END")) break;
        if (n >= ORC_NMAX) return -1;
        strncpy(m->species_names[n], a, 20);
        m->species_names[n][20] = 0;
        n++;
    }
    m->n_species = n;
    strcpy(m->species_names[n], "M");
    f->pos = 0;
    return 0;
}

/* chemical_reaction_parser (chemical_properties_class.f90:453-635) */
static void reaction_parser(const orc_mech *m, const char *reaction, const char *sign,
                            int *l1, int *l2, int *l3, int *r1, int *r2, int *r3,
                            int *ls, int *rs, int *unknown) {
    char left[160], right[160], spec1[160], rest[160], spec2[160], spec3[160];
    *l1 = *l2 = *l3 = *r1 = *r2 = *r3 = 0;
    *ls = *rs = 0;
    *unknown = 0;
    const char *pos = strstr(reaction, sign);
    size_t plen = (size_t)(pos - reaction);
    memcpy(left, reaction, plen);
    left[plen] = 0;
    size_t skip = strcmp(sign, "=") == 0 ? 1 : (strcmp(sign, "<=") == 0 ? 3 : 2);
    const char *rp = pos + skip;
    if (plen + skip > strlen(reaction)) rp = reaction + strlen(reaction);
    strncpy(right, rp, sizeof right - 1);
    right[sizeof right - 1] = 0;
    /* character(len=20) truncation of r_left1/r_right1 */
    left[20 < strlen(left) ? 20 : strlen(left)] = 0;
    right[20 < strlen(right) ? 20 : strlen(right)] = 0;

    for (int side = 0; side < 2; side++) {
        const char *s = side == 0 ? left : right;
        int *a1 = side == 0 ? l1 : r1, *a2 = side == 0 ? l2 : r2, *a3 = side == 0 ? l3 : r3;
        int *sum = side == 0 ? ls : rs;
        int twox = 0;
        const char *plus = strchr(s, '+');
        if (!plus) {
            if (s[0] == '2') {
                *a1 = specie_index(m, s + 1);
                *a2 = *a1;
                *sum = 2;
            } else {
                *a1 = specie_index(m, s);
                *sum = 1;
            }
            if (*a1 == 0) *unknown = 1;
        } else {
            size_t k = (size_t)(plus - s);
            memcpy(spec1, s, k);
            spec1[k] = 0;
            if (spec1[0] == '2') {
                *a1 = specie_index(m, spec1 + 1);
                *a2 = *a1;
                *sum = 2;
                twox = 1;
            } else {
                *a1 = specie_index(m, spec1);
                *sum = 1;
            }
            if (*a1 == 0) *unknown = 1;
            strcpy(rest, plus + 1);
            const char *plus2 = strchr(rest, '+');
            if (!plus2) {
                if (rest[0] == '2') {
                    *a2 = specie_index(m, rest + 1);
                    *a3 = *a2;
                    *sum = 3;
                    if (*a2 == 0) *unknown = 1;
                } else if (twox) {
                    *a3 = specie_index(m, rest);
                    *sum = 3;
                    if (*a3 == 0) *unknown = 1;
                } else {
                    *a2 = specie_index(m, rest);
                    *sum = 2;
                    if (*a2 == 0) *unknown = 1;
                }
            } else {
                size_t k2 = (size_t)(plus2 - rest);
                memcpy(spec2, rest, k2);
                spec2[k2] = 0;
                *a2 = specie_index(m, spec2);
                if (*a2 == 0) *unknown = 1;
                strcpy(spec3, plus2 + 1);
                *a3 = specie_index(m, spec3);
                if (*a3 == 0) *unknown = 1;
                *sum = 3;
            }
        }
    }
}

/* strip "(+M)" as the reference does: string(1:p-1)//string(p+4:len_trim-4) */
static void strip_falloff(char *s, size_t p /* 0-based */) {
    char out[160];
    size_t L = strlen(s);
    size_t k = 0;
    for (size_t i = 0; i < p && k < sizeof out - 1; i++) out[k++] = s[i];
    /* Fortran string(p+4 : L-4), 1-based p = p0+1 -> 0-based [p0+4, L-4) */
    for (size_t i = p + 4; i + 4 < L && k < sizeof out - 1; i++) out[k++] = s[i];
    out[k] = 0;
    strcpy(s, out);
}

static int classify(const char *s) {
    int r_type = 0;
    if (strchr(s, '=')) r_type = 1;
    if (strstr(s, "=>")) r_type = 2;
    if (strstr(s, "<=")) r_type = 3;
    return r_type;
}

static const char *sign_of(int r_type) {
    return r_type == 1 ? "=" : (r_type == 2 ? "=>" : "<=");
}

/* read_chemical_reactions_number (chemical_properties_class.f90:222-287) */
static int count_reactions(recfile *f, const orc_mech *m) {
    char tok[256];
    f->pos = 0;
    for (;;) {
        if (!ld_read_string(f, tok, sizeof tok)) return -1;
        if (fstr_eq(tok, "REACTIONS")) break;
    }
    int n = 0;
    for (;;) {
        if (!ld_read_string(f, tok, sizeof tok)) break;
        tok[150] = 0;
        char *fo = strstr(tok, "(+M)");
        if (fo) strip_falloff(tok, (size_t)(fo - tok));
        int r_type = classify(tok);
        if (r_type == 0) continue;
        int a, b, c, d, e, g, ls, rs, us;
        reaction_parser(m, tok, sign_of(r_type), &a, &b, &c, &d, &e, &g, &ls, &rs, &us);
        if (us) continue;
        n++;
    }
    f->pos = 0;
    return n;
}

/* READ(u,*) string, x1..xk from the current position; returns number of
 * reals read (sets *err nonzero if a conversion fails or EOF) */
static int ld_read_string_reals(recfile *f, char *str, size_t cap, double *x, int k, int *err) {
    ldscan s = {f, NULL, f->pos};
    char tok[256];
    *err = 0;
    int r = ld_next(&s, tok, sizeof tok);
    if (r != 1) { *err = r == 0 ? -1 : 0; return 0; }
    strncpy(str, tok, cap - 1);
    str[cap - 1] = 0;
    for (int i = 0; i < k; i++) {
        r = ld_next(&s, tok, sizeof tok);
        if (r != 1) { *err = r == 0 ? -1 : 0; return i; }
        if (fortran_real(tok, &x[i]) != 0) { *err = 1; return i; }
    }
    return k;
}

/* read_chemical_reactions_properties (chemical_properties_class.f90:289-451) */
static int read_reactions(recfile *f, orc_mech *m) {
    char tok[256];
    f->pos = 0;
    for (;;) {
        if (!ld_read_string(f, tok, sizeof tok)) return -1;
        if (fstr_eq(tok, "REACTIONS")) break;
    }
    int nr = 0;
    int enhanced = 0;
    int error = 0;
    for (;;) {
        if (!ld_read_string(f, tok, sizeof tok)) break;
        tok[150] = 0;
        int third_body = strstr(tok, "+M") != NULL;
        char *fo = strstr(tok, "(+M)");
        int falloff = fo != NULL;
        if (falloff) {
            strip_falloff(tok, (size_t)(fo - tok));
            enhanced = 1;
        }
        int r_type = classify(tok);
        if (r_type == 0) continue;
        int l1, l2, l3, r1, r2, r3, ls, rs, us;
        reaction_parser(m, tok, sign_of(r_type), &l1, &l2, &l3, &r1, &r2, &r3, &ls, &rs, &us);
        if (us) continue;
        if (nr >= m->n_reactions) return -1;
        int r = nr++;
        if (r_type == 2) {
            m->reaction_type[r] = third_body ? 6 : 5;
        } else {
            m->reaction_type[r] = third_body ? 1 : 0;
        }
        if (third_body) enhanced = 1;
        m->coeffs[0][r][0] = ls; m->coeffs[0][r][1] = l1; m->coeffs[0][r][2] = l2; m->coeffs[0][r][3] = l3;
        m->coeffs[1][r][0] = rs; m->coeffs[1][r][1] = r1; m->coeffs[1][r][2] = r2; m->coeffs[1][r][3] = r3;

        rf_backspace(f);
        double v[4];
        char s2[256];
        ld_read_string_reals(f, s2, sizeof s2, v, 3, &error);
        m->A[r] = v[0]; m->beta[r] = v[1]; m->E_act[r] = v[2];

        if (falloff) {
            error = ld_read_string(f, s2, sizeof s2) ? 0 : -1;
            if (fstr_eq(s2, "LOW")) {
                m->reaction_type[r] = 2;
                if (r_type == 2) m->reaction_type[r] = 7;
                rf_backspace(f);
                ld_read_string_reals(f, s2, sizeof s2, v, 3, &error);
                m->A_low[r] = v[0]; m->beta_low[r] = v[1]; m->E_act_low[r] = v[2];
            }
            error = ld_read_string(f, s2, sizeof s2) ? 0 : -1;
            if (fstr_eq(s2, "TROE")) {
                m->reaction_type[r] = 3;
                if (r_type == 2) m->reaction_type[r] = 7;
                rf_backspace(f);
                /* a list-directed read assigns the items read before an
                 * error; the others keep their value (zero from the
                 * allocation, chemical_properties_class.f90:156).  ZHANG.txt:27
                 * gives three TROE parameters: the read runs into the next
                 * record, fails there and consumes it. */
                const int got = ld_read_string_reals(f, s2, sizeof s2, v, 4, &error);
                for (int q = 0; q < got && q < 4; q++) m->troe[r][q] = v[q];
            } else {
                rf_backspace(f);
            }
        }

        if (error == 0) {
            char eff[256];
            error = ld_read_string(f, eff, sizeof eff) ? 0 : -1;
            if (error != 0) eff[0] = 0;
            eff[150] = 0;
            if (strchr(eff, '/') && enhanced) {
                /* species/value/ pairs */
                char buf[160];
                strncpy(buf, eff, sizeof buf - 1);
                buf[sizeof buf - 1] = 0;
                for (;;) {
                    /* adjtrim_length = len_trim(string) */
                    size_t L = strlen(buf);
                    while (L > 0 && buf[L - 1] == ' ') L--;
                    if (L == 0) break;
                    char *d1 = strchr(buf, '/');
                    if (!d1) {
                        /* index() = 0: string(1:-1) is empty, string(1:) kept */
                        d1 = buf - 1;
                    }
                    char name[160];
                    size_t nl = (size_t)(d1 - buf);
                    if (d1 < buf) nl = 0;
                    memcpy(name, buf, nl);
                    name[nl] = 0;
                    char *nm = name;
                    while (*nm == ' ') nm++;
                    int k = specie_index(m, nm);
                    char rest[160];
                    strcpy(rest, d1 + 1);
                    char *d2 = strchr(rest, '/');
                    if (k > 0) {
                        char num[160];
                        size_t ln = d2 ? (size_t)(d2 - rest) : 0;
                        memcpy(num, rest, ln);
                        num[ln] = 0;
                        double val;
                        if (fortran_real(num, &val) == 0) m->eff[r][k - 1] = val;
                    }
                    if (!d2) { buf[0] = 0; break; }
                    memmove(buf, d2 + 1, strlen(d2 + 1) + 1);
                }
            } else {
                rf_backspace(f);
            }
        }
    }
    f->pos = 0;
    return 0;
}

/* get_a_coeffs (thermophysical_properties_class.f90:1226-1311) */
static int get_a_coeffs(recfile *f, const char *name, double a[2][7]) {
    char tok[256];
    for (int s = 0; s < 2; s++)
        for (int i = 0; i < 7; i++) a[s][i] = 0.0;
    f->pos = 0;
    int found = 0;
    for (;;) {
        if (!ld_read_string(f, tok, sizeof tok)) break;
        tok[100] = 0;
        if (fstr_eq(tok, "END")) break;
        if (fstr_eq(tok, name)) {
            found = 1;
            int num = 0;
            int i1 = 1, i2 = 2;
            const char *cls = "-+E0123456789.";
            while (num < 16) {
                if (f->pos >= f->n) return -1;
                char line[101];
                strncpy(line, f->lines[f->pos++], 100);
                line[100] = 0;
                int prev = -1;
                int beginning = 1;
                int len = (int)strlen(line);
                while (len > 0 && line[len - 1] == ' ') len--;
                for (int i = 1; i <= len; i++) {
                    const char *q = strchr(cls, line[i - 1]);
                    int indx = (q && line[i - 1]) ? (int)(q - cls) + 1 : 0;
                    int boundary = ((indx == 0) && (prev > 0)) ||
                                   ((indx == 1) && ((prev != 3) && (prev > 0))) ||
                                   ((indx != 0) && (i == len));
                    if (boundary) {
                        if (num == 5 || num == 11) {
                            num = num + 1;
                        } else if (num == 16) {
                            break;
                        } else {
                            char nb[128];
                            int e = (i != len) ? i - 1 : i;
                            int L = e - beginning + 1;
                            if (L < 0) L = 0;
                            if (L > 120) L = 120;
                            memcpy(nb, line + beginning - 1, (size_t)L);
                            nb[L] = 0;
                            num = num + 1;
                            double v;
                            if (fortran_real(nb, &v) != 0) return -2;
                            a[i2 - 1][i1 - 1] = v;
                            i1 = i1 + 1;
                            if (num == 8) {
                                i1 = 1;
                                i2 = 1;
                            }
                        }
                        beginning = i;
                    }
                    prev = indx;
                }
            }
        }
    }
    f->pos = 0;
    return found ? 0 : 1;
}

/* get_specie_molar_mass (thermophysical_properties_class.f90:1313-1341) */
static int get_molar_mass(recfile *f, const char *name, double *w) {
    f->pos = 0;
    *w = 0.0;
    for (;;) {
        char s[256];
        double v;
        int err;
        if (f->pos >= f->n) return -1;
        int got = ld_read_string_reals(f, s, sizeof s, &v, 1, &err);
        if (err != 0 || got != 1) return -1;
        if (fstr_eq(s, name)) { *w = v; break; }
    }
    f->pos = 0;
    return 0;
}

int orc_load_mechanism(const char *mech_path, const char *thermo_path,
                       const char *molar_path, double eff_default,
                       const char *eact_units, orc_mech *out) {
    memset(out, 0, sizeof *out);
    recfile mf, tf, wf;
    if (rf_open(&mf, mech_path)) return 1;
    if (read_species(&mf, out)) { rf_close(&mf); return 2; }
    int nr = count_reactions(&mf, out);
    if (nr < 0 || nr > ORC_RMAX) { rf_close(&mf); return 3; }
    out->n_reactions = nr;
    for (int r = 0; r < nr; r++)
        for (int k = 0; k < out->n_species; k++) out->eff[r][k] = eff_default;
    if (read_reactions(&mf, out)) { rf_close(&mf); return 4; }
    rf_close(&mf);

    double coef;
    if (strcmp(eact_units, "J.mol") == 0) coef = 1.0;
    else if (strcmp(eact_units, "kJ.mol") == 0) coef = 1000.0;
    else if (strcmp(eact_units, "cal.mol") == 0) coef = R_GASE_J / R_GASE_CAL;
    else if (strcmp(eact_units, "kcal.mol") == 0) coef = R_GASE_J / R_GASE_CAL * 1000.0;
    else return 5;
    for (int r = 0; r < nr; r++) {
        int cl = out->coeffs[0][r][0];
        if (cl == 2) out->A[r] = out->A[r] * 1.0e-06;
        if (cl == 3) out->A[r] = out->A[r] * 1.0e-12;
        if (cl + 1 == 2) out->A_low[r] = out->A_low[r] * 1.0e-06;
        if (cl + 1 == 3) out->A_low[r] = out->A_low[r] * 1.0e-12;
        out->E_act[r] = out->E_act[r] * coef;
        out->E_act_low[r] = out->E_act_low[r] * coef;
    }

    if (rf_open(&tf, thermo_path)) return 6;
    if (rf_open(&wf, molar_path)) { rf_close(&tf); return 7; }
    for (int k = 0; k < out->n_species; k++) {
        char name[11];
        strncpy(name, out->species_names[k], 10); /* character(len=10) dummy */
        name[10] = 0;
        double a[2][7];
        if (get_a_coeffs(&tf, name, a) < 0) { rf_close(&tf); rf_close(&wf); return 8; }
        for (int s = 0; s < 2; s++)
            for (int i = 0; i < 7; i++) out->a_coeffs[k][s][i] = a[s][i] * R_GASE_J;
        if (get_molar_mass(&wf, name, &out->molar_mass[k])) { rf_close(&tf); rf_close(&wf); return 9; }
    }
    rf_close(&tf);
    rf_close(&wf);
    return 0;
}


/* get_transport_properties (thermophysical_properties_class.f90:1379-1414):
 * the first record is a header; then READ(u,*) name, geometry, eps/k_B,
 * sigma [Angstrom] until the name matches (an unreadable record or the end of
 * the file stops the reference's program).  sigma is returned in nm. */
static int get_transport(recfile *f, const char *name, double *eps, double *sigma) {
    f->pos = 0;
    *eps = 0.0;
    *sigma = 0.0;
    char hdr[256];
    if (!ld_read_string(f, hdr, sizeof hdr)) return -1;
    for (;;) {
        ldscan sc = {f, NULL, f->pos};
        char tok[4][256];
        for (int i = 0; i < 4; i++)
            if (ld_next(&sc, tok[i], sizeof tok[i]) != 1) return -1;
        char *end;
        strtol(tok[1], &end, 10);
        if (*end != 0 || end == tok[1]) return -1;
        double e, sg;
        if (fortran_real(tok[2], &e) || fortran_real(tok[3], &sg)) return -1;
        if (fstr_eq(tok[0], name)) {
            *eps = e;
            *sigma = sg * 0.1;
            break;
        }
    }
    f->pos = 0;
    return 0;
}

int orc_load_transport(const orc_mech *m, const char *transport_path, orc_transport *out) {
    memset(out, 0, sizeof *out);
    recfile tf;
    if (rf_open(&tf, transport_path)) return 1;
    const int N = m->n_species;
    out->n_species = N;
    for (int k = 0; k < N; k++) {
        char name[11];
        strncpy(name, m->species_names[k], 10); /* character(len=10) dummy */
        name[10] = 0;
        if (get_transport(&tf, name, &out->well_depth[k], &out->collision_diameter[k])) {
            rf_close(&tf);
            return 2;
        }
    }
    rf_close(&tf);
    /* initialize_binary_diffusivity_constants (:1343-1377) */
    const double *W = m->molar_mass, *sg = out->collision_diameter;
    for (int i = 0; i < N - 1; i++) {
        if (W[i] <= 0.0 || sg[i] <= 0.0) continue;
        for (int j = i + 1; j < N; j++) {
            if (W[j] <= 0.0 || sg[j] <= 0.0) continue;
            double red = 0.5 * (sg[i] + sg[j]);
            red = red * red;
            const double inv_mu = (W[i] + W[j]) / (W[i] * W[j]);
            out->bdc[i][j] = 0.00001 * 0.595 * sqrt(inv_mu) / red;
            out->bdc[j][i] = out->bdc[i][j];
        }
    }
    return 0;
}
