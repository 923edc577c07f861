/*
 * eb2_control.c -- ControlFile.txt reader of libeuler_b200.
 *
 * Accepts the reference's control-file format and keys (src/RP_FVM.c:382-589,
 * sample ControlFile.txt): `key: value` lines, '#' comment lines, the
 * reference's defaults for missing keys, its test-case names, and its
 * warnings on stderr for unknown keys, unknown case names and invalid
 * Recon_Accur / Characteriz values.  The reference exits when the file cannot
 * be opened; this returns EB2_EARG instead.  As in the reference, the values
 * of Recon_Accur and Characteriz are parsed and reported but the solver's
 * reconstruction is set separately (eb2_set_reconstruction).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/euler_b200.h"

/* TestCase2D names accepted by ReadControlFile (src/RP_FVM.c:436-477), with
 * their enumerator values (include/Golbal.h:8-30). */
static const struct {
    const char *name;
    int value;
} kCaseNames[] = {
    {"Precision_Test", 0},         {"1D_Sod_Shocktube", 1},    {"1D_Contact_Wave", 2},
    {"1D_Shock_Impact", 3},        {"1D_Impact_Wall", 4},      {"1D_Double_Rarefaction", 5},
    {"1D_Noh_Problem", 6},         {"2D_Riemann_Case1", 7},    {"2D_Riemann_Case2", 8},
    {"2D_Riemann_Case3", 9},       {"2D_Riemann_Case4", 10},   {"2D_Riemann_Case5", 11},
    {"Taylor_Green_Vortex", 12},   {"Gaussian_Pulse", 13},     {"Kelvin_Helmholtz", 14},
    {"Rayleigh_Taylor", 15},       {"Double_Mach_Reflection", 16},
    {"Odd_Even_Decoupling", 19},   {"Backward_Step", 20},      {"Blast_Wave", 17},
    {"2D_Noh_Problem", 18},
};

static void trim_spaces(char **s) {
    char *p = *s;
    while (*p == ' ') p++;
    size_t n = strlen(p);
    while (n > 0 && p[n - 1] == ' ') p[--n] = 0;
    *s = p;
}

static int truthy(const char *v) { return strcmp(v, "true") == 0 || strcmp(v, "1") == 0; }

static void set_defaults(eb2_control *c) {
    memset(c, 0, sizeof(*c));
    c->test_case = 15; /* Rayleigh_Taylor */
    c->L_nx = 100;
    c->L_ny = 400;
    c->Time_ADM = 3;
    c->scheme = 1;
    c->M_gamma = 1.4;
    c->Source = 0;
    c->Gravity = 1.0;
    c->CFL = 0.4;
    c->Tmax = 1.0;
    c->Control_Compution = 0;
    c->Control_output = 2;
    c->Recon_Accur = 2;
    c->Characteriz = 0;
    snprintf(c->output_dir, sizeof c->output_dir, "%s", "/mnt/d/Desktop/RP_FVM/data");
}

static void apply(eb2_control *c, const char *k, const char *v) {
    if (strcmp(k, "TestCase") == 0) {
        for (size_t n = 0; n < sizeof kCaseNames / sizeof kCaseNames[0]; n++)
            if (strcmp(v, kCaseNames[n].name) == 0) {
                c->test_case = kCaseNames[n].value;
                return;
            }
        fprintf(stderr, "Warning: Unknown test case '%s', using default Rayleigh_Taylor\n", v);
    } else if (strcmp(k, "L_nx") == 0) {
        c->L_nx = atoi(v);
    } else if (strcmp(k, "L_ny") == 0) {
        c->L_ny = atoi(v);
    } else if (strcmp(k, "Time_ADM") == 0) {
        c->Time_ADM = atoi(v);
    } else if (strcmp(k, "scheme") == 0) {
        c->scheme = atoi(v);
    } else if (strcmp(k, "M_gamma") == 0) {
        c->M_gamma = atof(v);
    } else if (strcmp(k, "Source") == 0) {
        c->Source = truthy(v);
    } else if (strcmp(k, "Gravity") == 0) {
        c->Gravity = atof(v);
    } else if (strcmp(k, "CFL") == 0) {
        c->CFL = atof(v);
    } else if (strcmp(k, "Tmax") == 0) {
        c->Tmax = atof(v);
    } else if (strcmp(k, "Control_Compution") == 0) {
        c->Control_Compution = atoi(v);
    } else if (strcmp(k, "Control_output") == 0) {
        c->Control_output = atoi(v);
    } else if (strcmp(k, "output_dir") == 0) {
        snprintf(c->output_dir, sizeof c->output_dir, "%s", v);
    } else if (strcmp(k, "Recon_Accur") == 0) {
        int r = atoi(v);
        if (r == 1 || r == 2 || r == 3 || r == 5) {
            c->Recon_Accur = r;
        } else {
            fprintf(stderr,
                    "Warning: Invalid Recon_Accur value %d. Valid values are 1, 2, 3, 5. "
                    "Using default 2.\n", r);
            c->Recon_Accur = 2;
        }
    } else if (strcmp(k, "Characteriz") == 0) {
        if (truthy(v)) {
            c->Characteriz = 1;
        } else if (strcmp(v, "false") == 0 || strcmp(v, "0") == 0) {
            c->Characteriz = 0;
        } else {
            fprintf(stderr, "Warning: Invalid Characteriz value '%s'. Using default false.\n", v);
            c->Characteriz = 0;
        }
    } else {
        fprintf(stderr, "Warning: Unknown parameter '%s' in control file\n", k);
    }
}

int eb2_read_control_file(const char *path, eb2_control *out) {
    if (!path || !out) return EB2_EARG;
    FILE *fp = fopen(path, "r");
    if (!fp) {
        fprintf(stderr, "Error: Cannot open control file %s\n", path);
        return EB2_EARG;
    }
    set_defaults(out);
    char line[256], key[100], value[150];
    while (fgets(line, sizeof line, fp)) {
        if (line[0] == '#' || line[0] == '\n' || line[0] == '\r') continue;
        line[strcspn(line, "\n")] = 0;
        line[strcspn(line, "\r")] = 0;
        if (sscanf(line, "%99[^:]: %149[^\n]", key, value) != 2) continue;
        char *k = key, *v = value;
        trim_spaces(&k);
        trim_spaces(&v);
        apply(out, k, v);
    }
    fclose(fp);
    return EB2_OK;
}
