/* Constants of fx_math.h, written by gen_fx_math_consts.py (do not edit): each the stated
   real number rounded to the stated number of significant bits. */
#ifndef FX_MATH_CONSTS_H
#define FX_MATH_CONSTS_H

#define FXM_INV_LN2_32 0x1.71547652b82fep+5 /* 32 / ln 2 */
#define FXM_LN2_32_1 0x1.62e42fefa0000p-6 /* ln 2 / 32, first 36 bits */
#define FXM_LN2_32_2 0x1.cf79abc9e0000p-45 /* ln 2 / 32, next 36 bits */
#define FXM_LN2_32_3 0x1.d9cc01f97b57ap-84 /* ln 2 / 32, the rest */
#define FXM_EXP_C3 0x1.5555555555555p-3 /* 1/3! */
#define FXM_EXP_C4 0x1.5555555555555p-5 /* 1/4! */
#define FXM_EXP_C5 0x1.1111111111111p-7 /* 1/5! */
#define FXM_EXP_C6 0x1.6c16c16c16c17p-10 /* 1/6! */
#define FXM_EXP_C7 0x1.a01a01a01a01ap-13 /* 1/7! */
/* 2^(j/32), j = 0..31, as double-double: high and low parts */
#define FXM_EXP2_HI_INIT 0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0, 0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0, 0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0, 0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0, 0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0, 0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0, 0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0, 0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0
#define FXM_EXP2_LO_INIT 0x0.0p+0, 0x1.d73e2a475b465p-55, 0x1.8a62e4adc610bp-54, -0x1.6c51039449b3ap-54, -0x1.19041b9d78a76p-55, 0x1.e016e00a2643cp-54, 0x1.9b07eb6c70573p-54, 0x1.612e8afad1255p-55, 0x1.6f46ad23182e4p-55, -0x1.63aeabf42eae2p-54, 0x1.ada0911f09ebcp-55, 0x1.89b7a04ef80d0p-59, 0x1.d4397afec42e2p-56, -0x1.07abe1db13cadp-55, 0x1.6324c054647adp-54, -0x1.383c17e40b497p-54, -0x1.bdd3413b26456p-54, -0x1.16e4786887a99p-55, -0x1.41577ee04992fp-55, -0x1.d4c1dd41532d8p-54, 0x1.6e9f156864b27p-54, -0x1.75fc781b57ebcp-57, 0x1.c7c46b071f2bep-56, -0x1.d2f6edb8d41e1p-54, 0x1.7a1cd345dcc81p-54, -0x1.5584f7e54ac3bp-56, 0x1.11065895048ddp-55, 0x1.503cbd1e949dbp-56, 0x1.2ed02d75b3707p-55, -0x1.1a5cd4f184b5cp-54, -0x1.e9c23179c2893p-54, 0x1.9d3e12dd8a18bp-54
#define FXM_LN2_HI 0x1.62e42fefa3800p-1 /* ln 2, first 42 bits */
#define FXM_LN2_LO 0x1.ef35793c76730p-45 /* ln 2, the rest */
#define FXM_SQRT2 0x1.6a09e667f3bcdp+0 /* sqrt 2 */
#define FXM_LOG_A1 0x1.5555555555555p-1 /* 2/3 */
#define FXM_LOG_A2 0x1.999999999999ap-2 /* 2/5 */
#define FXM_LOG_A3 0x1.2492492492492p-2 /* 2/7 */
#define FXM_LOG_A4 0x1.c71c71c71c71cp-3 /* 2/9 */
#define FXM_LOG_A5 0x1.745d1745d1746p-3 /* 2/11 */
#define FXM_LOG_A6 0x1.3b13b13b13b14p-3 /* 2/13 */
#define FXM_LOG_A7 0x1.1111111111111p-3 /* 2/15 */
#define FXM_LOG_A8 0x1.e1e1e1e1e1e1ep-4 /* 2/17 */
#define FXM_LOG_A9 0x1.af286bca1af28p-4 /* 2/19 */
#define FXM_LOG_A10 0x1.8618618618618p-4 /* 2/21 */
#define FXM_LOG_A11 0x1.642c8590b2164p-4 /* 2/23 */
#define FXM_LOG_A12 0x1.47ae147ae147bp-4 /* 2/25 */
#define FXM_LOG_A13 0x1.2f684bda12f68p-4 /* 2/27 */
#define FXM_TWO_OVER_PI 0x1.45f306dc9c883p-1 /* 2 / pi */
#define FXM_PIO2_1 0x1.921fb54400000p+0 /* pi / 2, first 33 bits */
#define FXM_PIO2_2 0x1.0b4611a600000p-34 /* pi / 2, next 33 bits */
#define FXM_PIO2_3 0x1.3198a2e037073p-69 /* pi / 2, the rest */
#define FXM_COS_C2 0x1.5555555555555p-5 /* (-1)^2/4! */
#define FXM_COS_C3 -0x1.6c16c16c16c17p-10 /* (-1)^3/6! */
#define FXM_COS_C4 0x1.a01a01a01a01ap-16 /* (-1)^4/8! */
#define FXM_COS_C5 -0x1.27e4fb7789f5cp-22 /* (-1)^5/10! */
#define FXM_COS_C6 0x1.1eed8eff8d898p-29 /* (-1)^6/12! */
#define FXM_COS_C7 -0x1.93974a8c07c9dp-37 /* (-1)^7/14! */
#define FXM_COS_C8 0x1.ae7f3e733b81fp-45 /* (-1)^8/16! */
#define FXM_COS_C9 -0x1.6827863b97d97p-53 /* (-1)^9/18! */
#define FXM_COS_C10 0x1.e542ba4020225p-62 /* (-1)^10/20! */
#define FXM_SIN_S1 -0x1.5555555555555p-3 /* (-1)^1/3! */
#define FXM_SIN_S2 0x1.1111111111111p-7 /* (-1)^2/5! */
#define FXM_SIN_S3 -0x1.a01a01a01a01ap-13 /* (-1)^3/7! */
#define FXM_SIN_S4 0x1.71de3a556c734p-19 /* (-1)^4/9! */
#define FXM_SIN_S5 -0x1.ae64567f544e4p-26 /* (-1)^5/11! */
#define FXM_SIN_S6 0x1.6124613a86d09p-33 /* (-1)^6/13! */
#define FXM_SIN_S7 -0x1.ae7f3e733b81fp-41 /* (-1)^7/15! */
#define FXM_SIN_S8 0x1.952c77030ad4ap-49 /* (-1)^8/17! */
#define FXM_SIN_S9 -0x1.2f49b46814157p-57 /* (-1)^9/19! */
#define FXM_COS_C2_LO 0x1.5555555555555p-59 /* 1/24 - FXM_COS_C2 */
#define FXM_SIN_S1_LO -0x1.5555555555555p-57 /* -1/6 - FXM_SIN_S1 */

#endif
