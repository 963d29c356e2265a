/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The table_approximated mode of the chemistry step, restated from
 * computing_module/src/current_build/chemical_kinetics_solver.f90:
 *   write_chemical_kinetics_table   :542-607
 *   read_chemical_kinetics_table    :608-650
 *   interpolate_chemical_kinetics   :651-685
 *   solve_chemical_kinetics, the branches this mode takes:
 *     no rate constants (:250-252), conc_in = Y (:256-262),
 *     interpolation instead of DDRIV3 (:314-315),
 *     Y_prod = conc_out * W / dt (:323-325), E_f_prod from conc_out (:334-335).
 * The table file is formatted text: one header record, then one record per
 * row written with the edit descriptor (N+1)E14.7 (T, then the N values of
 * Y_prod2 along the tabulated row).
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define T_REF 298.15 /* global_data.f90:38 */

/* Fortran Ew.d output with w = 14, d = 7 (0.dddddddE+xx; the exponent letter
 * is dropped when |exponent| > 99), right-justified, blank-padded. */
void orc_format_e14_7(double x, char out[15]) {
    char body[32];
    if (isnan(x)) {
        snprintf(out, 15, "%14s", "NaN");
        return;
    }
    if (isinf(x)) {
        snprintf(out, 15, "%14s", x < 0 ? "-Infinity" : "Infinity");
        return;
    }
    const int neg = signbit(x) != 0;
    const double ax = fabs(x);
    char digits[8];
    int e10 = 0;
    if (ax == 0.0) {
        memcpy(digits, "0000000", 8);
        e10 = 0;
    } else {
        char tmp[40];
        snprintf(tmp, sizeof tmp, "%.6e", ax); /* d.dddddde+XX, correctly rounded */
        digits[0] = tmp[0];
        memcpy(digits + 1, tmp + 2, 6);
        digits[7] = '\0';
        e10 = atoi(strchr(tmp, 'e') + 1) + 1; /* 0.ddddddd scaling */
    }
    const int ae = e10 < 0 ? -e10 : e10;
    if (ae <= 99)
        snprintf(body, sizeof body, "%s0.%sE%c%02d", neg ? "-" : "", digits, e10 < 0 ? '-' : '+', ae);
    else
        snprintf(body, sizeof body, "%s0.%s%c%03d", neg ? "-" : "", digits, e10 < 0 ? '-' : '+', ae);
    const size_t L = strlen(body); /* at most 14: sign, "0.", 7 digits, 4 exponent characters */
    memset(out, ' ', 14);
    memcpy(out + 14 - L, body, L);
    out[14] = '\0';
}

/* Fortran Ew.d input with d = 7 on one field of `len` characters: blanks are
 * ignored (BLANK = NULL), an all-blank field is zero, a mantissa without a
 * decimal point has its last d digits as the fraction, and the exponent is
 * E/D followed by a signed integer or a bare signed integer.  Returns 0 and
 * stores the value, or -1 on a malformed field. */
int orc_parse_e14_7(const char *field, int len, double *value) {
    char s[64];
    int n = 0;
    for (int i = 0; i < len && field[i] != '\0' && field[i] != '\n' && field[i] != '\r'; ++i)
        if (field[i] != ' ' && field[i] != '\t' && n < 62) s[n++] = field[i];
    s[n] = '\0';
    if (n == 0) {
        *value = 0.0;
        return 0;
    }
    int p = 0, neg = 0;
    if (s[p] == '+' || s[p] == '-') neg = s[p++] == '-';
    char mant[64];
    int m = 0, point = -1, ndig = 0;
    while (isdigit((unsigned char)s[p]) || s[p] == '.') {
        if (s[p] == '.') {
            if (point >= 0) return -1;
            point = ndig;
        } else {
            mant[m++] = s[p];
            ++ndig;
        }
        ++p;
    }
    if (ndig == 0) return -1;
    mant[m] = '\0';
    long ex = 0;
    if (s[p] == 'E' || s[p] == 'e' || s[p] == 'D' || s[p] == 'd') ++p;
    if (s[p] != '\0') {
        int eneg = 0;
        if (s[p] == '+' || s[p] == '-') eneg = s[p++] == '-';
        else if (!(s[p - 1] == 'E' || s[p - 1] == 'e' || s[p - 1] == 'D' || s[p - 1] == 'd')) return -1;
        if (!isdigit((unsigned char)s[p])) return -1;
        while (isdigit((unsigned char)s[p])) ex = ex * 10 + (s[p++] - '0');
        if (s[p] != '\0') return -1;
        if (eneg) ex = -ex;
    }
    /* digits with the decimal point at `point` (or d = 7 from the right) */
    const long frac = point >= 0 ? ndig - point : 7;
    char buf[96];
    snprintf(buf, sizeof buf, "%s0.%se%ld", neg ? "-" : "", mant, ex - frac + ndig);
    *value = strtod(buf, NULL);
    return 0;
}

static int blank_record(const char *line) {
    for (const char *c = line; *c; ++c)
        if (!isspace((unsigned char)*c)) return 0;
    return 1;
}

/* read_chemical_kinetics_table (:608-650).  The row count is the number of
 * records a list-directed read of a character variable accepts (records with
 * a non-blank character) less the header; after the header, that many
 * records are read with (N+1)E14.7 (a short or blank record reads as zeros).
 * T_t[i], Y_t[k*capacity + i].  With T_t == NULL only *rows is set.
 * Returns 0, -1 (unreadable), -2 (malformed field), -3 (no row). */
int orc_table_read(const char *path, int n_species, long capacity, double *T_t, double *Y_t, long *rows) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[8192];
    long records = 0;
    while (fgets(line, sizeof line, f))
        if (!blank_record(line)) ++records;
    const long size = records - 1;
    *rows = size < 0 ? 0 : size;
    if (size < 1) {
        fclose(f);
        return -3;
    }
    if (!T_t) {
        fclose(f);
        return 0;
    }
    rewind(f);
    while (fgets(line, sizeof line, f))
        if (!blank_record(line)) break; /* the header */
    for (long i = 0; i < size && i < capacity; ++i) {
        if (!fgets(line, sizeof line, f)) line[0] = '\0';
        const size_t L = strlen(line);
        for (int q = 0; q <= n_species; ++q) {
            char fld[15];
            memset(fld, ' ', 14);
            fld[14] = '\0';
            const size_t at = (size_t)q * 14;
            for (size_t c = 0; c < 14 && at + c < L; ++c) fld[c] = line[at + c];
            double v;
            if (orc_parse_e14_7(fld, 14, &v) != 0) {
                fclose(f);
                return -2;
            }
            if (q == 0) T_t[i] = v;
            else Y_t[(size_t)(q - 1) * (size_t)capacity + (size_t)i] = v;
        }
    }
    fclose(f);
    return 0;
}

/* write_chemical_kinetics_table (:542-607) on one row of cells (the
 * reference's T%cells(i,1,1)): row arrays indexed by the Fortran index i in
 * [lb, ub] (T_row[i - lb], Y_prod2_row[k*(ub-lb+1) + i - lb]); lo..hi is the
 * interior.  min_index is the first interior i with 300.5 < T < 310 (0 when
 * none), max_index the first interior i holding the largest T above 0 (0
 * when none); rows min_index..max_index are written.  names: species names
 * for the header.  Returns 0, -1 (cannot write), -4 (rows outside [lb, ub]). */
int orc_table_write(const char *path, int n_species, const char (*names)[21], int lb, int ub, int lo, int hi,
                    const double *T_row, const double *Y_prod2_row) {
    double max_T = 0.0;
    int min_index = 0, max_index = 0;
    for (int i = lo; i <= hi; ++i) {
        const double t = T_row[i - lb];
        if (t > 300.5 && t < 310.0 && min_index == 0) min_index = i;
        if (t > max_T) {
            max_index = i;
            max_T = t;
        }
    }
    if (min_index <= max_index && (min_index < lb || max_index > ub)) return -4;
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    fputs("T", f);
    for (int k = 0; k < n_species; ++k) fprintf(f, "  r(%s)", names[k]);
    fputc('\n', f);
    const long ext = (long)ub - lb + 1;
    for (int i = min_index; i <= max_index; ++i) {
        char fld[15];
        orc_format_e14_7(T_row[i - lb], fld);
        fputs(fld, f);
        for (int k = 0; k < n_species; ++k) {
            orc_format_e14_7(Y_prod2_row[(long)k * ext + (i - lb)], fld);
            fputs(fld, f);
        }
        fputc('\n', f);
    }
    return fclose(f) == 0 ? 0 : -1;
}

/* interpolate_chemical_kinetics (:651-685): the last interval i with
 * T_t(i) <= T <= T_t(i+1) sets every species linearly in T (the reference's
 * operation order); below the first node every value is 0, above the last
 * the last row is taken; otherwise the values are left as they came in. */
static void interpolate(int N, long M, const double *T_t, const double *Y_t, double T, double *conc) {
    for (long i = 0; i < M - 1; ++i) {
        if (T >= T_t[i] && T <= T_t[i + 1]) {
            for (int k = 0; k < N; ++k)
                conc[k] = Y_t[(long)k * M + i + 1] * (T - T_t[i]) / (T_t[i + 1] - T_t[i]) +
                          Y_t[(long)k * M + i] * (T - T_t[i + 1]) / (T_t[i] - T_t[i + 1]);
        }
    }
    if (T < T_t[0])
        for (int k = 0; k < N; ++k) conc[k] = 0.0;
    if (T > T_t[M - 1])
        for (int k = 0; k < N; ++k) conc[k] = Y_t[(long)k * M + M - 1];
}

/* The chemistry step in table_approximated mode over n cells (SoA Y[k*n+c];
 * table rows T_t[i], Y_t[k*M + i]).  Skip rule as the integrating mode:
 * zero sources, Y_prod2 untouched. */
int orc_table_step(const orc_mech *m, long M, const double *T_t, const double *Y_t, long n, double dt,
                   const double *T, const double *Y, const signed char *bc, double *Y_prod, double *Y_prod2,
                   double *E_f_prod, int n_threads) {
    const int N = m->n_species;
    if (M < 1) return -3;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
#else
    (void)n_threads;
#endif
    for (long c = 0; c < n; ++c) {
        const double Tc = T[c];
        if (!((Tc >= 305.0) && (bc == NULL || bc[c] == 0))) {
            for (int k = 0; k < N; k++) Y_prod[(long)k * n + c] = 0.0;
            E_f_prod[c] = 0.0;
            continue;
        }
        double conc_in[ORC_NMAX], conc_out[ORC_NMAX];
        for (int k = 0; k < N; ++k) {
            conc_in[k] = Y[(long)k * n + c]; /* mass fractions in this mode */
            conc_out[k] = conc_in[k];
        }
        interpolate(N, M, T_t, Y_t, Tc, conc_out);
        for (int k = 0; k < N; ++k) {
            const double W = m->molar_mass[k];
            if (W != 0.0) {
                Y_prod[(long)k * n + c] = conc_out[k] * W / dt;
                Y_prod2[(long)k * n + c] = conc_out[k] - conc_in[k];
            } else {
                Y_prod[(long)k * n + c] = conc_out[k] - conc_in[k];
            }
        }
        double E = 0.0;
        for (int k = 0; k < N; ++k) E = E - orc_specie_enthalpy(m, T_REF, k) * conc_out[k] / dt;
        E_f_prod[c] = E;
    }
    return 0;
}
