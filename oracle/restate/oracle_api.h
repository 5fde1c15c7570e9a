/*
 * Oracle test infrastructure: parameter structs and field identifiers shared
 * by the two CPU oracles,
 *   - oracle/_ref/libleniaref.so  : the reference's own lenia.cpp,
 *     reintegration.cpp, transposition.cpp and mesh.cpp compiled unmodified
 *     against shim headers (render.h's compile-time grid, 32x32x32), and
 *   - oracle/_build/liblenia_oracle.so : the C restatement (lenia_oracle.c),
 *     whose grid size and kernel count are runtime values.
 * Tests drive both through ctypes.  Nothing in the product library uses it.
 *
 * The parameter set is the reference's mutable globals (main.cpp:27-66,
 * main.cpp:304, render.h:347-361, render.h:486-492).
 */
#ifndef LENIA_ORACLE_API_H
#define LENIA_ORACLE_API_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_MAX_BETA 12
#define ORA_MAX_CHANNELS 4

typedef struct {
    int width;   /* x and z extent (GRID_WIDTH) */
    int height;  /* y extent (GRID_HEIGHT) */
    int channels;
    float timestep;
    float theta_a;
    float n_alpha;   /* N: read but unused by the reference (Q3) */
    float s_norm;
    float gta;
    float sta;
    float v_damp;
    float v_beta;    /* unused by the reference */
    float iso_value;
    float sigma;     /* off_table.sigma */
    float dd;        /* off_table.dd, used as (int) */
    int alpha_mode;
    int growth_type;   /* 0 NOGROWTH, 1 RT, 2 TRANSPOSITION */
    int mode_type;     /* 0 SRT, 1 RT, 2 ADV */
    int sobel_border;  /* 0 TORUS, 1 WALL, 2 NONE */
    int border;        /* 0 TORUS, 1 WALL, 2 NONE */
    int gradient_mode; /* 0 CENTRAL_DIFF, 1 SOBEL */
    int adv_vel;
    int mu_vel;
    int blur_central_diff;
    int osc_la;
    int osc_flow;
    int osc_div_flow;
    int osc_vel;
    float osc_la_amt;
    float osc_flow_amt;
    float osc_div_flow_amt;
    int asymptotic[ORA_MAX_CHANNELS];
    int soft_clip[ORA_MAX_CHANNELS];
    int rt_all_channels; /* 0: reference (SRT/RT move channels 0-2 only, Q7) */
    int alpha_index_fix; /* 0: reference (PREALPHA/GA channel offsets, Q20) */
    int exact_bell;      /* 0: reference growth table (Q1); 1: bell(u, m, s) per cell */
} ora_params;

typedef struct {
    int radius;
    int beta_size;
    float b[ORA_MAX_BETA];
    float r_a;
    float m;
    float s;
    float h;
    int c0;
    int c1;
} ora_kernel;

/* Field identifiers; every field is returned unpadded, channel-major,
 * x fastest (IDX of render.h:334).  Vector fields are three blocks x, y, z. */
enum {
    ORA_A = 0,      /* GRID */
    ORA_V = 1,      /* V_x, V_y, V_z  (3*C*N) */
    ORA_GA = 2,
    ORA_SUM = 3,    /* N */
    ORA_H = 4,
    ORA_U_SUM = 5,
    ORA_BACK = 6,
    ORA_NA = 7,     /* 3*N */
    ORA_NU = 8,     /* 3*C*N */
    ORA_PREALPHA = 9,
    ORA_ALPHA = 10,
    ORA_F = 11,     /* 3*C*N */
    ORA_MU = 12,    /* 3*C*N */
    ORA_TT = 13,
    ORA_U_S = 14,
    ORA_SUM_S = 15, /* N */
    ORA_U = 16,     /* K*N: Re(U_k)/N, the value the growth LUT is indexed with */
    ORA_H_RB = 17,
    ORA_U_SUM_RB = 18,
    ORA_RBB = 19,
    ORA_NFIELDS = 20
};

/* Step events in the reference's order (render.h:181-197). */
enum {
    ORA_EV_FFT = 0, ORA_EV_FFT_MT, ORA_EV_BLUR, ORA_EV_TSB, ORA_EV_SOBEL_ONE, ORA_EV_SOBEL_TWO,
    ORA_EV_F, ORA_EV_MU, ORA_EV_TB, ORA_EV_REINTEGRATION, ORA_EV_TRM, ORA_EV_TMB, ORA_EV_MAX
};

#ifdef __cplusplus
}
#endif
#endif
