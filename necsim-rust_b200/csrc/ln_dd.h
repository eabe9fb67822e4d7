/*
 * ln_dd.h -- a natural logarithm for (0, 1] evaluated in double-double
 * arithmetic and rounded once.  The same C source compiles for the host
 * (C or C++) and the device (CUDA) and gives the same bits on both: every
 * operation is an IEEE-754 round-to-nearest +, -, *, / or an fma whose
 * result is exact or correctly rounded, written out explicitly so that no
 * compiler may contract or reorder it (on the device through the __d*_rn /
 * __fma_rn intrinsics, on the host as plain operators in a translation unit
 * built with -ffp-contract=off, and the C library's correctly rounded fma).
 * It serves the exponential event-time sampler (`-ln(U(0,1]) / lambda`),
 * whose event times must agree bit for bit between the GPU and its checker.
 *
 * Method (table-driven reduction, as in Tang 1990, then a Taylor series):
 *   x = m * 2^k with m in [sqrt(1/2), sqrt(2)), so x near 1 keeps k = 0;
 *   i = floor((m - 359/512) * 256) picks an interval of width 1/256 and
 *   c_i ~ 1 / centre_i (c = 1 exactly on the interval centred on 1), so
 *   r = m * c_i - 1 is exact as a double-double (fma product error, Sterbenz
 *   subtraction) with |r| < 2^-8.49;
 *   ln x = k ln 2 - ln c_i + ln(1 + r), ln(1 + r) = r P(r),
 *   P(r) = sum_{n=1..12} (-1)^(n+1) r^(n-1) / n (truncation < 2^-105 |r|):
 *   terms 1..6 in double-double, evaluated in powers of r^2 to keep the
 *   dependent chain short, terms 7..12 in double (their rounding errors
 *   stay below 2^-106 |r|).
 *   ln 2, -ln c_i (gen_ln_table.py, from 60-digit decimal arithmetic) and the
 *   coefficients 1/3, 1/5, 1/6 are double-double roundings of the exact values.
 * The relative error before the final rounding is below ~2^-98, so the
 * result is the correctly rounded logarithm except for inputs within
 * ~2^-45 ulp of a rounding boundary (none met in tests).
 */
#ifndef NECSIM_LN_DD_H
#define NECSIM_LN_DD_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define NECSIM_DD_FN static __host__ __device__ __forceinline__
#else
#define NECSIM_DD_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define NECSIM_DD_ADD(a, b) __dadd_rn((a), (b))
#define NECSIM_DD_SUB(a, b) __dsub_rn((a), (b))
#define NECSIM_DD_MUL(a, b) __dmul_rn((a), (b))
#define NECSIM_DD_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define NECSIM_DD_ADD(a, b) ((a) + (b))
#define NECSIM_DD_SUB(a, b) ((a) - (b))
#define NECSIM_DD_MUL(a, b) ((a) * (b))
#define NECSIM_DD_FMA(a, b, c) fma((a), (b), (c))
#endif

/* generated by gen_ln_table.py: c_i and -ln(c_i) as hi + lo */
#define NECSIM_LN_TABLE_N 183
#define NECSIM_LN_TABLE_C \
    {0x1.6c16c16c16c17p+0, 0x1.6a13cd1537290p+0, 0x1.6816816816817p+0, 0x1.661ec6a5122f9p+0, \
    0x1.642c8590b2164p+0, 0x1.623fa77016240p+0, 0x1.6058160581606p+0, 0x1.5e75bb8d015e7p+0, \
    0x1.5c9882b931057p+0, 0x1.5ac056b015ac0p+0, 0x1.58ed2308158edp+0, 0x1.571ed3c506b3ap+0, \
    0x1.5555555555555p+0, 0x1.5390948f40febp+0, 0x1.51d07eae2f815p+0, 0x1.5015015015015p+0, \
    0x1.4e5e0a72f0539p+0, 0x1.4cab88725af6ep+0, 0x1.4afd6a052bf5bp+0, 0x1.49539e3b2d067p+0, \
    0x1.47ae147ae147bp+0, 0x1.460cbc7f5cf9ap+0, 0x1.446f86562d9fbp+0, 0x1.42d6625d51f87p+0, \
    0x1.4141414141414p+0, 0x1.3fb013fb013fbp+0, 0x1.3e22cbce4a902p+0, 0x1.3c995a47babe7p+0, \
    0x1.3b13b13b13b14p+0, 0x1.3991c2c187f63p+0, 0x1.3813813813814p+0, 0x1.3698df3de0748p+0, \
    0x1.3521cfb2b78c1p+0, 0x1.33ae45b57bcb2p+0, 0x1.323e34a2b10bfp+0, 0x1.30d190130d190p+0, \
    0x1.2f684bda12f68p+0, 0x1.2e025c04b8097p+0, 0x1.2c9fb4d812ca0p+0, 0x1.2b404ad012b40p+0, \
    0x1.29e4129e4129ep+0, 0x1.288b01288b013p+0, 0x1.27350b8812735p+0, 0x1.25e22708092f1p+0, \
    0x1.2492492492492p+0, 0x1.23456789abcdfp+0, 0x1.21fb78121fb78p+0, 0x1.20b470c67c0d9p+0, \
    0x1.1f7047dc11f70p+0, 0x1.1e2ef3b3fb874p+0, 0x1.1cf06ada2811dp+0, 0x1.1bb4a4046ed29p+0, \
    0x1.1a7b9611a7b96p+0, 0x1.19453808ca29cp+0, 0x1.1811811811812p+0, 0x1.16e0689427379p+0, \
    0x1.15b1e5f75270dp+0, 0x1.1485f0e0acd3bp+0, 0x1.135c81135c811p+0, 0x1.12358e75d3033p+0, \
    0x1.1111111111111p+0, 0x1.0fef010fef011p+0, 0x1.0ecf56be69c90p+0, 0x1.0db20a88f4696p+0, \
    0x1.0c9714fbcda3bp+0, 0x1.0b7e6ec259dc8p+0, 0x1.0a6810a6810a7p+0, 0x1.0953f39010954p+0, \
    0x1.0842108421084p+0, 0x1.073260a47f7c6p+0, 0x1.0624dd2f1a9fcp+0, 0x1.05197f7d73404p+0, \
    0x1.0410410410410p+0, 0x1.03091b51f5e1ap+0, 0x1.0204081020408p+0, 0x1.0101010101010p+0, \
    0x1.0000000000000p+0, 0x1.fe01fe01fe020p-1, 0x1.fc07f01fc07f0p-1, 0x1.fa11caa01fa12p-1, \
    0x1.f81f81f81f820p-1, 0x1.f6310aca0dbb5p-1, 0x1.f44659e4a4271p-1, 0x1.f25f644230ab5p-1, \
    0x1.f07c1f07c1f08p-1, 0x1.ee9c7f8458e02p-1, 0x1.ecc07b301ecc0p-1, 0x1.eae807aba01ebp-1, \
    0x1.e9131abf0b767p-1, 0x1.e741aa59750e4p-1, 0x1.e573ac901e574p-1, 0x1.e3a9179dc1a73p-1, \
    0x1.e1e1e1e1e1e1ep-1, 0x1.e01e01e01e01ep-1, 0x1.de5d6e3f8868ap-1, 0x1.dca01dca01dcap-1, \
    0x1.dae6076b981dbp-1, 0x1.d92f2231e7f8ap-1, 0x1.d77b654b82c34p-1, 0x1.d5cac807572b2p-1, \
    0x1.d41d41d41d41dp-1, 0x1.d272ca3fc5b1ap-1, 0x1.d0cb58f6ec074p-1, 0x1.cf26e5c44bfc6p-1, \
    0x1.cd85689039b0bp-1, 0x1.cbe6d9601cbe7p-1, 0x1.ca4b3055ee191p-1, 0x1.c8b265afb8a42p-1, \
    0x1.c71c71c71c71cp-1, 0x1.c5894d10d4986p-1, 0x1.c3f8f01c3f8f0p-1, 0x1.c26b5392ea01cp-1, \
    0x1.c0e070381c0e0p-1, 0x1.bf583ee868d8bp-1, 0x1.bdd2b899406f7p-1, 0x1.bc4fd65883e7bp-1, \
    0x1.bacf914c1bad0p-1, 0x1.b951e2b18ff23p-1, 0x1.b7d6c3dda338bp-1, 0x1.b65e2e3beee05p-1, \
    0x1.b4e81b4e81b4fp-1, 0x1.b37484ad806cep-1, 0x1.b2036406c80d9p-1, 0x1.b094b31d922a4p-1, \
    0x1.af286bca1af28p-1, 0x1.adbe87f94905ep-1, 0x1.ac5701ac5701bp-1, 0x1.aaf1d2f87ebfdp-1, \
    0x1.a98ef606a63bep-1, 0x1.a82e65130e159p-1, 0x1.a6d01a6d01a6dp-1, 0x1.a574107688a4ap-1, \
    0x1.a41a41a41a41ap-1, 0x1.a2c2a87c51ca0p-1, 0x1.a16d3f97a4b02p-1, 0x1.a01a01a01a01ap-1, \
    0x1.9ec8e951033d9p-1, 0x1.9d79f176b682dp-1, 0x1.9c2d14ee4a102p-1, 0x1.9ae24ea5510dap-1, \
    0x1.999999999999ap-1, 0x1.9852f0d8ec0ffp-1, 0x1.970e4f80cb872p-1, 0x1.95cbb0be377aep-1, \
    0x1.948b0fcd6e9e0p-1, 0x1.934c67f9b2ce6p-1, 0x1.920fb49d0e229p-1, 0x1.90d4f120190d5p-1, \
    0x1.8f9c18f9c18fap-1, 0x1.8e6527af1373fp-1, 0x1.8d3018d3018d3p-1, 0x1.8bfce8062ff3ap-1, \
    0x1.8acb90f6bf3aap-1, 0x1.899c0f601899cp-1, 0x1.886e5f0abb04ap-1, 0x1.87427bcc092b9p-1, \
    0x1.8618618618618p-1, 0x1.84f00c2780614p-1, 0x1.83c977ab2beddp-1, 0x1.82a4a0182a4a0p-1, \
    0x1.8181818181818p-1, 0x1.8060180601806p-1, 0x1.7f405fd017f40p-1, 0x1.7e225515a4f1dp-1, \
    0x1.7d05f417d05f4p-1, 0x1.7beb3922e017cp-1, 0x1.7ad2208e0ecc3p-1, 0x1.79baa6bb6398bp-1, \
    0x1.78a4c8178a4c8p-1, 0x1.77908119ac60dp-1, 0x1.767dce434a9b1p-1, 0x1.756cac201756dp-1, \
    0x1.745d1745d1746p-1, 0x1.734f0c541fe8dp-1, 0x1.724287f46debcp-1, 0x1.713786d9c7c09p-1, \
    0x1.702e05c0b8170p-1, 0x1.6f26016f26017p-1, 0x1.6e1f76b4337c7p-1, 0x1.6d1a62681c861p-1, \
    0x1.6c16c16c16c17p-1, 0x1.6b1490aa31a3dp-1, 0x1.6a13cd1537290p-1}
#define NECSIM_LN_TABLE_LHI \
    {-0x1.68ac83e9c6a15p-2, -0x1.630030b3aac48p-2, -0x1.5d5bddf595f31p-2, -0x1.57bf753c8d1fbp-2, \
    -0x1.522ae0738a3d7p-2, -0x1.4c9e09e172c3dp-2, -0x1.4718dc271c41cp-2, -0x1.419b423d5e8c6p-2, \
    -0x1.3c25277333183p-2, -0x1.36b6776be1116p-2, -0x1.314f1e1d35ce3p-2, -0x1.2bef07cdc9355p-2, \
    -0x1.269621134db91p-2, -0x1.214456d0eb8d5p-2, -0x1.1bf99635a6b95p-2, -0x1.16b5ccbacfb73p-2, \
    -0x1.1178e8227e47ap-2, -0x1.0c42d676162e2p-2, -0x1.07138604d5864p-2, -0x1.01eae5626c691p-2, \
    -0x1.f991c6cb3b37ap-3, -0x1.ef5ade4dcffe5p-3, -0x1.e530effe71013p-3, -0x1.db13db0d48941p-3, \
    -0x1.d1037f2655e7bp-3, -0x1.c6ffbc6f00f71p-3, -0x1.bd087383bd8aap-3, -0x1.b31d8575bce3bp-3, \
    -0x1.a93ed3c8ad9e5p-3, -0x1.9f6c407089663p-3, -0x1.95a5adcf70182p-3, -0x1.8beafeb38fe8fp-3, \
    -0x1.823c16551a3c0p-3, -0x1.7898d85444c74p-3, -0x1.6f0128b756ab9p-3, -0x1.6574ebe8c1339p-3, \
    -0x1.5bf406b543db0p-3, -0x1.527e5e4a1b58dp-3, -0x1.4913d8333b563p-3, -0x1.3fb45a59928cap-3, \
    -0x1.365fcb0159014p-3, -0x1.2d1610c86813dp-3, -0x1.23d712a49c201p-3, -0x1.1aa2b7e23f729p-3, \
    -0x1.1178e8227e47ap-3, -0x1.08598b59e3a07p-3, -0x1.fe89139dbd565p-4, -0x1.ec739830a1126p-4, \
    -0x1.da7276384469ep-4, -0x1.c885801bc4b20p-4, -0x1.b6ac88dad5b1dp-4, -0x1.a4e7640b1bc38p-4, \
    -0x1.9335e5d594988p-4, -0x1.8197e2f40e3f0p-4, -0x1.700d30aeac0e8p-4, -0x1.5e95a4d9791cdp-4, \
    -0x1.4d3115d207eacp-4, -0x1.3bdf5a7d1ee5ep-4, -0x1.2aa04a44717a1p-4, -0x1.1973bd1465561p-4, \
    -0x1.08598b59e3a06p-4, -0x1.eea31c006b87cp-5, -0x1.ccb73cdddb2d0p-5, -0x1.aaef2d0fb1108p-5, \
    -0x1.894aa149fb34bp-5, -0x1.67c94f2d4bb65p-5, -0x1.466aed42de3f9p-5, -0x1.252f32f8d1840p-5, \
    -0x1.0415d89e74440p-5, -0x1.c63d2ec14aad7p-6, -0x1.8492528c8cac5p-6, -0x1.432a925980cbcp-6, \
    -0x1.0205658935837p-6, -0x1.82448a388a283p-7, -0x1.010157588de69p-7, -0x1.0080559588b25p-8, \
    0x0.0p+0, 0x1.ff00aa2b10ba0p-9, 0x1.fe02a6b106799p-8, 0x1.7dc475f810a69p-7, \
    0x1.fc0a8b0fc03c4p-7, 0x1.3cea44346a584p-6, 0x1.7b91b07d5b126p-6, 0x1.b9fc027af919ap-6, \
    0x1.f829b0e7832f8p-6, 0x1.1b0d98923d97fp-5, 0x1.39e87b9febd68p-5, 0x1.58a5bafc8e4d3p-5, \
    0x1.77458f632dcffp-5, 0x1.95c830ec8e3f2p-5, 0x1.b42dd711971b9p-5, 0x1.d276b8adb0b56p-5, \
    0x1.f0a30c01162a8p-5, 0x1.075983598e471p-4, 0x1.16536eea37ae3p-4, 0x1.253f62f0a1417p-4, \
    0x1.341d7961bd1d0p-4, 0x1.42edcbea646eep-4, 0x1.51b073f06183cp-4, 0x1.60658a93750c4p-4, \
    0x1.6f0d28ae56b4ep-4, 0x1.7da766d7b12d0p-4, 0x1.8c345d6319b23p-4, 0x1.9ab42462033aep-4, \
    0x1.a926d3a4ad562p-4, 0x1.b78c82bb0eda0p-4, 0x1.c5e548f5bc743p-4, 0x1.d4313d66cb35dp-4, \
    0x1.e27076e2af2eap-4, 0x1.f0a30c01162a4p-4, 0x1.fec9131dbeabcp-4, 0x1.0671512ca596fp-3, \
    0x1.0d77e7cd08e5bp-3, 0x1.14785846742acp-3, 0x1.1b72ad52f67a2p-3, 0x1.2266f190a5acdp-3, \
    0x1.29552f81ff521p-3, 0x1.303d718e47fd5p-3, 0x1.371fc201e8f75p-3, 0x1.3dfc2b0ecc62ap-3, \
    0x1.44d2b6ccb7d1cp-3, 0x1.4ba36f39a55e5p-3, 0x1.526e5e3a1b438p-3, 0x1.59338d9982085p-3, \
    0x1.5ff3070a793d6p-3, 0x1.66acd4272ad51p-3, 0x1.6d60fe719d21bp-3, 0x1.740f8f54037a3p-3, \
    0x1.7ab890210d907p-3, 0x1.815c0a14357e9p-3, 0x1.87fa06520c911p-3, 0x1.8e928de886d41p-3, \
    0x1.9525a9cf456b6p-3, 0x1.9bb362e7dfb85p-3, 0x1.a23bc1fe2b561p-3, 0x1.a8becfc882f19p-3, \
    0x1.af3c94e80bff3p-3, 0x1.b5b519e8fb5a6p-3, 0x1.bc286742d8cd4p-3, 0x1.c2968558c18c2p-3, \
    0x1.c8ff7c79a9a20p-3, 0x1.cf6354e09c5ddp-3, 0x1.d5c216b4fbb94p-3, 0x1.dc1bca0abec7bp-3, \
    0x1.e27076e2af2e8p-3, 0x1.e8c0252aa5a60p-3, 0x1.ef0adcbdc5935p-3, 0x1.f550a564b7b37p-3, \
    0x1.fb9186d5e3e29p-3, 0x1.00e6c45ad501dp-2, 0x1.0402594b4d041p-2, 0x1.071b85fcd590dp-2, \
    0x1.0a324e27390e2p-2, 0x1.0d46b579ab74bp-2, 0x1.1058bf9ae4ad4p-2, 0x1.136870293a8b0p-2, \
    0x1.1675cababa60fp-2, 0x1.1980d2dd4236fp-2, 0x1.1c898c16999fbp-2, 0x1.1f8ff9e48a2f3p-2, \
    0x1.22941fbcf7966p-2, 0x1.2596010df763ap-2, 0x1.2895a13de86a4p-2, 0x1.2b9303ab89d25p-2, \
    0x1.2e8e2bae11d31p-2, 0x1.31871c9544185p-2, 0x1.347dd9a987d56p-2, 0x1.3772662bfd85cp-2, \
    0x1.3a64c556945eap-2, 0x1.3d54fa5c1f710p-2, 0x1.404308686a7e4p-2, 0x1.432ef2a04e813p-2, \
    0x1.4618bc21c5ec2p-2, 0x1.49006804009d0p-2, 0x1.4be5f957778a1p-2, 0x1.4ec9732600269p-2, \
    0x1.51aad872df82ep-2, 0x1.548a2c3add263p-2, 0x1.5767717455a6cp-2, 0x1.5a42ab0f4cfe2p-2, \
    0x1.5d1bdbf5809cap-2, 0x1.5ff3070a793d4p-2, 0x1.62c82f2b9c796p-2}
#define NECSIM_LN_TABLE_LLO \
    {0x1.acd8a9145ff44p-57, -0x1.ee0c6728fffccp-56, -0x1.d5f75b9a23ae4p-59, 0x1.2908d15f88b63p-57, \
    -0x1.3840b263acb43p-56, 0x1.123615b147a5fp-58, -0x1.d8fb4c14c56eep-56, -0x1.5b7648704e721p-58, \
    -0x1.152d81af5713ap-56, 0x1.324f0e8838590p-58, -0x1.22966f61a3c23p-56, 0x1.22dad7fd86088p-56, \
    -0x1.e0efadd9db02ap-56, 0x1.50a2dca28b3edp-58, 0x1.e9575c2124912p-56, -0x1.56fbd28b40935p-56, \
    -0x1.b8ce2d07f1cb7p-56, 0x1.5a74e18a8bb85p-56, 0x1.24e912b16ec8bp-60, -0x1.d9f5bd0b5b348p-57, \
    -0x1.ecca0cdf30143p-58, -0x1.7754d2238f75fp-58, 0x1.f7627ef82f3f0p-57, 0x1.8af715b0349a4p-57, \
    0x1.3f3adb7b71cbcp-58, 0x1.ae58b2c57a4a5p-57, 0x1.1165504ad749ep-59, 0x1.0d4eace1aa537p-59, \
    -0x1.bcafa9de97202p-57, 0x1.52979a7e86605p-57, -0x1.8a16283fdbd1cp-57, 0x1.54aae92cd0b87p-59, \
    -0x1.6dcd318f4187ep-57, -0x1.be3dbaf3ec804p-60, 0x1.37967087859b9p-59, -0x1.c5961e173bc82p-57, \
    0x1.1f5b44c0df7f7p-61, 0x1.b8d4b411cadffp-60, 0x1.0d5604930f137p-58, 0x1.d87e6a354d057p-57, \
    -0x1.bea08d2dca256p-57, -0x1.d997036941a6dp-60, -0x1.51c7e9efae297p-57, -0x1.6e44389934420p-57, \
    0x1.0e63a5f01c693p-58, 0x1.fd7009902bf32p-57, 0x1.ac9f4215f9394p-58, -0x1.eea033743f95bp-58, \
    -0x1.401fa71733017p-58, 0x1.5c734aa6598fcp-58, 0x1.002bf768e52d0p-58, 0x1.9b5ca203e4259p-58, \
    0x1.478a85704ccb7p-58, 0x1.230690020895fp-59, -0x1.a36a677b4c8b2p-59, 0x1.4c78ba3a3baf6p-58, \
    -0x1.da7d0b1e10b2fp-60, -0x1.f52eda76b68acp-60, -0x1.aea2c72d05c08p-58, 0x1.7aac1b3d35680p-58, \
    0x1.dd7009902bf32p-58, 0x1.7c9f9276f6cd8p-60, 0x1.e48fb0500efd5p-59, -0x1.68d4eed0b82aep-59, \
    0x1.2ba0b44cfaee5p-59, -0x1.0413e6505e5f9p-59, 0x1.9badefe942718p-60, -0x1.ae021b67a9ba8p-61, \
    -0x1.c05cf1d753621p-59, -0x1.8fe7acbca131dp-63, 0x1.d192d0619fa68p-60, 0x1.8cdaf39004193p-60, \
    -0x1.27c8e8416e717p-60, -0x1.04b16137f0970p-62, -0x1.46662d417cecep-62, -0x1.f96638cf63675p-62, \
    0x0.0p+0, 0x1.2821ad5a6d357p-63, -0x1.e44b7e3711e7fp-67, 0x1.74944bc161072p-61, \
    -0x1.83092c5964281p-62, -0x1.865ad48159d00p-61, -0x1.6d80ab38e9430p-62, -0x1.90ae69229dc86p-60, \
    0x1.33e3f04f1ef25p-60, -0x1.74d7444dd6241p-59, -0x1.5bfa937f551b7p-59, -0x1.cab8569c56e40p-64, \
    0x1.8d3ca87b92968p-63, 0x1.eb41d00a417e9p-60, 0x1.0a34531f67db5p-59, 0x1.078f14c95ff53p-59, \
    0x1.85f325c5bbacdp-59, 0x1.006d2999e22dcp-58, 0x1.2189705cf74cap-58, 0x1.1f6d34e01d981p-61, \
    -0x1.3599f227becbbp-58, -0x1.511583653349bp-58, -0x1.5b61c65e5741ap-58, -0x1.f108b1d8436d3p-59, \
    -0x1.20db323097324p-59, 0x1.a2240644d7da2p-59, -0x1.294d2f5668495p-58, -0x1.a099e1c184e8ep-59, \
    -0x1.d7a16eab1e2adp-59, -0x1.3ef0e61f9b03cp-58, 0x1.2eb0bf7c0b0d9p-59, 0x1.b90dd951d90fap-58, \
    -0x1.61578001e015ap-60, 0x1.8be64b8b7759bp-59, -0x1.5746b9981b36cp-58, -0x1.2f39b81479b67p-58, \
    0x1.9a5dc5e9030adp-57, 0x1.94409f1d3f83ap-60, -0x1.fbe7ee5c69946p-57, -0x1.dab840e7f6177p-57, \
    0x1.301771c407dc0p-57, -0x1.b5ae71f658247p-57, 0x1.e6cb62af18a02p-62, 0x1.ba62b8c13f7f4p-57, \
    0x1.7d3d950f87e23p-59, -0x1.f767e433c98aap-57, -0x1.546ff8a470d3ap-57, 0x1.8d16eaaba9419p-57, \
    -0x1.bc60efafc6f6cp-58, -0x1.9201c9c3d5165p-59, 0x1.d551d97132e87p-57, 0x1.6d9bf9d57b326p-58, \
    -0x1.1072534a57e7dp-57, 0x1.141b7f8c5fa9ep-58, -0x1.9f7fdbfa08d9ap-57, 0x1.2589eb96a6240p-59, \
    -0x1.26fb3e2b1d1dap-57, -0x1.51439c1ff83e7p-58, 0x1.24dc46c1ea664p-57, -0x1.a8c37918c39ebp-58, \
    0x1.a3398064df33ep-57, -0x1.d5d8023e61e5fp-57, 0x1.cfce744870f57p-58, 0x1.6108e3ae024acp-60, \
    -0x1.4f689f8434011p-57, 0x1.339a07d55b696p-57, -0x1.a37794d03657dp-58, 0x1.c698a33316dfbp-58, \
    -0x1.61578001e015ep-59, -0x1.dc074737f9135p-60, 0x1.e8637950dc20dp-57, -0x1.13a09202fe73dp-57, \
    0x1.355519b0de535p-57, -0x1.3b9568ff6feadp-57, -0x1.08ec217a5022dp-57, 0x1.08b83fcbdef40p-57, \
    0x1.bdcfde8061c03p-56, 0x1.21f640e1e5ec9p-56, 0x1.3f415699663ecp-63, 0x1.86cc531dba494p-57, \
    0x1.ce63eab883727p-61, -0x1.02c2e4f1b2eb9p-56, 0x1.9f1a39d500e3cp-56, -0x1.93fbf3418960dp-57, \
    -0x1.dbd7ac258a2bdp-58, -0x1.9eed8ae0ebd3cp-59, 0x1.7ad24c13f040fp-56, -0x1.85ad7f614ab51p-58, \
    -0x1.1e99b72bd7bf2p-57, -0x1.ea3598981366fp-57, -0x1.16ea62c048cfbp-56, 0x1.02a7589fba088p-57, \
    0x1.cbcd735d03424p-60, 0x1.53668e578d9cdp-58, -0x1.f79f6c1059cdbp-57, -0x1.83262e2b59206p-57, \
    -0x1.7a42642661c62p-61, -0x1.bff0d07c5df6dp-59, -0x1.4b366b609027ap-58, -0x1.1aa87d977dc5ep-56, \
    -0x1.d8db0a7cc1543p-56, -0x1.58ce7bf1846eep-56, -0x1.fb2a49af933e8p-57, -0x1.c6bcb7dee9a3dp-56, \
    -0x1.7dc9c7c23801fp-56, -0x1.063077d7e37b7p-56, -0x1.090a0dd59fe35p-58}

/* the reduction table, in device memory for the device and in host memory
 * for the host (one definition per translation unit that uses it) */
#if defined(__CUDACC__)
static __device__ const double necsim_ln_c_d[NECSIM_LN_TABLE_N] = NECSIM_LN_TABLE_C;
static __device__ const double necsim_ln_lhi_d[NECSIM_LN_TABLE_N] = NECSIM_LN_TABLE_LHI;
static __device__ const double necsim_ln_llo_d[NECSIM_LN_TABLE_N] = NECSIM_LN_TABLE_LLO;
#endif
static const double necsim_ln_c_h[NECSIM_LN_TABLE_N] = NECSIM_LN_TABLE_C;
static const double necsim_ln_lhi_h[NECSIM_LN_TABLE_N] = NECSIM_LN_TABLE_LHI;
static const double necsim_ln_llo_h[NECSIM_LN_TABLE_N] = NECSIM_LN_TABLE_LLO;
#if defined(__CUDA_ARCH__)
#define NECSIM_LN_C necsim_ln_c_d
#define NECSIM_LN_LHI necsim_ln_lhi_d
#define NECSIM_LN_LLO necsim_ln_llo_d
#else
#define NECSIM_LN_C necsim_ln_c_h
#define NECSIM_LN_LHI necsim_ln_lhi_h
#define NECSIM_LN_LLO necsim_ln_llo_h
#endif

typedef struct necsim_dd {
    double hi, lo;
} necsim_dd;

NECSIM_DD_FN necsim_dd necsim_dd_make(double hi, double lo) {
    necsim_dd r;
    r.hi = hi;
    r.lo = lo;
    return r;
}

/* a + b = s + e exactly (Knuth) */
NECSIM_DD_FN necsim_dd necsim_dd_two_sum(double a, double b) {
    const double s = NECSIM_DD_ADD(a, b);
    const double bb = NECSIM_DD_SUB(s, a);
    return necsim_dd_make(s, NECSIM_DD_ADD(NECSIM_DD_SUB(a, NECSIM_DD_SUB(s, bb)), NECSIM_DD_SUB(b, bb)));
}

/* a + b = s + e exactly when |a| >= |b| (Dekker) */
NECSIM_DD_FN necsim_dd necsim_dd_quick_two_sum(double a, double b) {
    const double s = NECSIM_DD_ADD(a, b);
    return necsim_dd_make(s, NECSIM_DD_SUB(b, NECSIM_DD_SUB(s, a)));
}

/* a * b = p + e exactly; the fma computes the exact residual */
NECSIM_DD_FN necsim_dd necsim_dd_two_prod(double a, double b) {
    const double p = NECSIM_DD_MUL(a, b);
    return necsim_dd_make(p, NECSIM_DD_FMA(a, b, -p));
}

NECSIM_DD_FN necsim_dd necsim_dd_add(necsim_dd a, necsim_dd b) {
    necsim_dd s = necsim_dd_two_sum(a.hi, b.hi);
    const necsim_dd t = necsim_dd_two_sum(a.lo, b.lo);
    s = necsim_dd_quick_two_sum(s.hi, NECSIM_DD_ADD(s.lo, t.hi));
    return necsim_dd_quick_two_sum(s.hi, NECSIM_DD_ADD(s.lo, t.lo));
}

NECSIM_DD_FN necsim_dd necsim_dd_mul(necsim_dd a, necsim_dd b) {
    const necsim_dd p = necsim_dd_two_prod(a.hi, b.hi);
    const double cross = NECSIM_DD_ADD(NECSIM_DD_MUL(a.hi, b.lo), NECSIM_DD_MUL(a.lo, b.hi));
    return necsim_dd_quick_two_sum(p.hi, NECSIM_DD_ADD(p.lo, cross));
}

/* a + b with one two-sum (Dekker's addition): relative error ~2^-104 as long
 * as a and b do not nearly cancel, which holds for every sum below (the
 * worst cancellation, -ln c + ln(1 + r) next to the interval centred on 1,
 * loses one bit) */
NECSIM_DD_FN necsim_dd necsim_dd_add_fast(necsim_dd a, necsim_dd b) {
    const necsim_dd s = necsim_dd_two_sum(a.hi, b.hi);
    return necsim_dd_quick_two_sum(s.hi, NECSIM_DD_ADD(s.lo, NECSIM_DD_ADD(a.lo, b.lo)));
}

/* a + b for a double b */
NECSIM_DD_FN necsim_dd necsim_dd_add_d(necsim_dd a, double b) {
    const necsim_dd s = necsim_dd_two_sum(a.hi, b);
    return necsim_dd_quick_two_sum(s.hi, NECSIM_DD_ADD(s.lo, a.lo));
}

/* a * b for a double b */
NECSIM_DD_FN necsim_dd necsim_dd_mul_d(necsim_dd a, double b) {
    const necsim_dd p = necsim_dd_two_prod(a.hi, b);
    return necsim_dd_quick_two_sum(p.hi, NECSIM_DD_ADD(p.lo, NECSIM_DD_MUL(a.lo, b)));
}

/* a * a */
NECSIM_DD_FN necsim_dd necsim_dd_sqr(necsim_dd a) {
    const necsim_dd p = necsim_dd_two_prod(a.hi, a.hi);
    return necsim_dd_quick_two_sum(p.hi, NECSIM_DD_ADD(p.lo, NECSIM_DD_MUL(NECSIM_DD_ADD(a.hi, a.hi), a.lo)));
}

/* ln(x) for normal doubles 0 < x <= 1, one rounding of a double-double */
NECSIM_DD_FN double necsim_ln(double x) {
    uint64_t bits;
    double m;
    int k, i;
    necsim_dd r, a, b, c, r2, p, base, res;
    double rh, r6, tail;
    if (x == 1.0) return 0.0;
    memcpy(&bits, &x, 8);
    k = (int)((bits >> 52) & 0x7ff) - 1022; /* x = m * 2^k, m in [0.5, 1) */
    bits = (bits & 0x000fffffffffffffULL) | 0x3fe0000000000000ULL;
    memcpy(&m, &bits, 8);
    if (m < 0.70710678118654752) { /* into [sqrt(1/2), sqrt(2)), exactly */
        m = NECSIM_DD_MUL(m, 2.0);
        k -= 1;
    }
    /* m - 359/512 is exact (both are multiples of ulp(m)), the scaling too */
    i = (int)NECSIM_DD_MUL(NECSIM_DD_SUB(m, 0.701171875), 256.0);
    /* r = m * c_i - 1 exactly: p + e = m * c_i, p - 1 exact (p within 2^-8 of 1) */
    r = necsim_dd_two_prod(m, NECSIM_LN_C[i]);
    r = necsim_dd_two_sum(NECSIM_DD_SUB(r.hi, 1.0), r.lo);
    /* k ln 2 - ln c_i, independent of the series (|k ln 2| >= 0.69 > 2 |ln c_i|
     * when k != 0) */
    base = necsim_dd_add_fast(necsim_dd_mul_d(necsim_dd_make(0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56),
                                              (double)k),
                              necsim_dd_make(NECSIM_LN_LHI[i], NECSIM_LN_LLO[i]));
    /* terms 7..12 in double: r^6 (1/7 - r/8 + r^2/9 - r^3/10 + r^4/11 - r^5/12) */
    rh = r.hi;
    tail = -0x1.5555555555555p-4;
    tail = NECSIM_DD_FMA(tail, rh, 0x1.745d1745d1746p-4);
    tail = NECSIM_DD_FMA(tail, rh, -0x1.999999999999ap-4);
    tail = NECSIM_DD_FMA(tail, rh, 0x1.c71c71c71c71cp-4);
    tail = NECSIM_DD_FMA(tail, rh, -0x1.0000000000000p-3);
    tail = NECSIM_DD_FMA(tail, rh, 0x1.2492492492492p-3);
    r6 = NECSIM_DD_MUL(rh, rh);
    r6 = NECSIM_DD_MUL(NECSIM_DD_MUL(r6, r6), r6);
    tail = NECSIM_DD_MUL(r6, tail);
    /* terms 1..6 in double-double: (1 - r/2) + r^2 ((1/3 - r/4) + r^2 (1/5 - r/6));
     * each sum adds a term at most 2^-6 the size of the other */
    a = necsim_dd_add_d(necsim_dd_make(NECSIM_DD_MUL(r.hi, -0.5), NECSIM_DD_MUL(r.lo, -0.5)), 1.0);
    b = necsim_dd_add_fast(necsim_dd_make(0x1.5555555555555p-2, 0x1.5555555555555p-56),
                           necsim_dd_make(NECSIM_DD_MUL(r.hi, -0.25), NECSIM_DD_MUL(r.lo, -0.25)));
    c = necsim_dd_add_fast(necsim_dd_make(0x1.999999999999ap-3, -0x1.999999999999ap-57),
                           necsim_dd_mul(necsim_dd_make(-0x1.5555555555555p-3, -0x1.5555555555555p-57), r));
    r2 = necsim_dd_sqr(r);
    p = necsim_dd_add_fast(a, necsim_dd_mul(r2, necsim_dd_add_fast(b, necsim_dd_mul(r2, c))));
    p = necsim_dd_add_d(p, tail);
    res = necsim_dd_add_fast(base, necsim_dd_mul(r, p));
    return NECSIM_DD_ADD(res.hi, res.lo);
}

#endif /* NECSIM_LN_DD_H */
