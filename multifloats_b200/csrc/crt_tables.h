// Generated by gen_crt_tables.py -- do not edit.
// Moduli of the CRT split form and their per-modulus constants.
#pragma once
#include <stdint.h>
#ifndef MF_TABLE
#define MF_TABLE static const
#endif
#define CRT_NMAX 36
MF_TABLE uint32_t crt_mod[36] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163, 157, 151, 149, 139, 137, 131, 127, 113, 109, 107, 103, 101, 97, 89};
MF_TABLE int crt_lg[37] = {0, 8, 15, 23, 31, 39, 47, 55, 63, 71, 79, 87, 94, 102, 110, 117, 125, 132, 140, 147, 155, 162, 170, 177, 184, 191, 198, 206, 213, 220, 226, 233, 240, 247, 253, 260, 266};
#ifdef __cplusplus
// host copy of crt_lg (workspace sizing)
static constexpr int crt_lg_host[37] = {0, 8, 15, 23, 31, 39, 47, 55, 63, 71, 79, 87, 94, 102, 110, 117, 125, 132, 140, 147, 155, 162, 170, 177, 184, 191, 198, 206, 213, 220, 226, 233, 240, 247, 253, 260, 266};
#endif
MF_TABLE uint32_t crt_digw[36][4] = {{0x00000001u, 0x00000000u, 0x00000000u, 0x00000000u},
    {0x01010101u, 0x01010101u, 0x01010101u, 0x00000101u},
    {0x1b090301u, 0xa6e2f651u, 0x2f64cdefu, 0x0000ad90u},
    {0x7d190501u, 0x403f717bu, 0x5be05e45u, 0x000010d1u},
    {0xf4510901u, 0x3d991094u, 0x51090137u, 0x000094f4u},
    {0x01f00f01u, 0x0f01f00fu, 0xf00f01f0u, 0x00000f01u},
    {0x96321101u, 0x3303d66eu, 0x715bb1a7u, 0x0000aa09u},
    {0x333f1701u, 0xc626cf08u, 0x02474a40u, 0x0000952eu},
    {0xf52a1b01u, 0x3d94fcbcu, 0xe6102b2cu, 0x000035f1u},
    {0x64bd1d01u, 0x960c6ecdu, 0xd6454168u, 0x00005aadu},
    {0x22e62101u, 0x0f290807u, 0x69403831u, 0x0000ca99u},
    {0x4e022701u, 0x5f08c304u, 0xca20e510u, 0x00009440u},
    {0xe5ab2d01u, 0x6460e633u, 0x242bc445u, 0x000069bcu},
    {0xb4413901u, 0x5605232eu, 0xe81f12b7u, 0x00002019u},
    {0xa4bf3b01u, 0xedf94658u, 0xa0e7353du, 0x0000c031u},
    {0xafac3f01u, 0xc1ff31abu, 0xcf555154u, 0x00003f01u},
    {0xdf174101u, 0xb4c705d4u, 0xa219e31au, 0x0000c302u},
    {0xdc0e4b01u, 0x031d270fu, 0x2d492a2cu, 0x000057c0u},
    {0x53164d01u, 0x4c5724cbu, 0x592b3dc9u, 0x0000f533u},
    {0x16e15301u, 0x24dd0ab3u, 0xfcb7b22fu, 0x0000cf0eu},
    {0x3e48b201u, 0xbd03d307u, 0x20151331u, 0x0000de09u},
    {0xd00aba01u, 0xb71609c1u, 0x2351b239u, 0x000018fbu},
    {0x2743c601u, 0x10cfc8c0u, 0x4bfce50eu, 0x0000012eu},
    {0x3b02d201u, 0xbe08df04u, 0x26201310u, 0x0000b540u},
    {0xdde8d601u, 0xd321caecu, 0x06c025d1u, 0x0000052eu},
    {0x3743ea01u, 0x1fdfbc29u, 0x1425f80du, 0x0000cee9u},
    {0x3b32ee01u, 0xcf38c022u, 0xeaf2103cu, 0x0000fcf1u},
    {0x2e24fa01u, 0x0b14d1f2u, 0xe9ee0341u, 0x0000d607u},
    {0x08040201u, 0x01c12010u, 0x10080402u, 0x0000c120u},
    {0xf9fc1e01u, 0x01311c10u, 0x10f9fc1eu, 0x0000311cu},
    {0x2d1b2601u, 0xfcd210deu, 0x1b2601d5u, 0x0000de2du},
    {0x2c342a01u, 0xf80a291du, 0xeee10cf1u, 0x00001bf9u},
    {0xd61c3201u, 0x200dd5d8u, 0xd4fbe1d0u, 0x000004dbu},
    {0x05f3d101u, 0x251924dfu, 0xf7ef18eau, 0x00001013u},
    {0xffdcdd01u, 0xdd012423u, 0x2423ffdcu, 0x0000dd01u},
    {0x0420f501u, 0x021027d4u, 0x0108e7eau, 0x000020f5u}};
MF_TABLE uint32_t crt_inv_bits[36] = {0x3b800000u, 0x3b808081u, 0x3b81848eu, 0x3b828cc0u, 0x3b84a9fau, 0x3b87f781u, 0x3b891ac7u, 0x3b8ca29cu, 0x3b8f177au, 0x3b905a38u, 0x3b92f114u, 0x3b97012eu, 0x3b9b4c70u, 0x3ba4a9cfu, 0x3ba655c4u, 0x3ba9c84au, 0x3bab8f6au, 0x3bb509e7u, 0x3bb70fbbu, 0x3bbd6910u, 0x3bc43730u, 0x3bc907dau, 0x3bd0b6a0u, 0x3bd901b2u, 0x3bdbeb62u, 0x3bebbdb3u, 0x3bef2eb7u, 0x3bfa232du, 0x3c010204u, 0x3c10fdbcu, 0x3c164fdau, 0x3c191f1au, 0x3c1f1166u, 0x3c2237c3u, 0x3c28e83fu, 0x3c381703u};  // float(1/m) bit patterns
MF_TABLE int crt_rlo[36] = {-128, -127, -126, -125, -123, -120, -119, -116, -114, -113, -111, -108, -105, -99, -98, -96, -95, -90, -89, -86, -83, -81, -78, -75, -74, -69, -68, -65, -63, -56, -54, -53, -51, -50, -48, -44};
MF_TABLE int crt_rhi[36] = {127, 127, 126, 125, 123, 120, 119, 116, 114, 113, 111, 108, 105, 99, 98, 96, 95, 90, 89, 86, 83, 81, 78, 75, 74, 69, 68, 65, 63, 56, 54, 53, 51, 50, 48, 44};
