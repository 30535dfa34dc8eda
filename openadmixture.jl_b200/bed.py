"""Minimal PLINK 1 binary genotype I/O (.bed/.bim/.fam), SNP-major.

The reference opens files through SnpArrays.SnpArray (driver.jl:144-145), which checks the
3-byte magic (0x6c 0x1b 0x01), takes I from the .fam line count and J from the .bim line
count, and exposes the packed column bytes as ``g.s.data`` (ceil(I/4) x J).  This module does
the same and returns the bytes as a numpy array of shape (J, ceil(I/4)) -- the same memory as
Julia's ceil(I/4) x J column-major matrix.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

BED_MAGIC = bytes([0x6C, 0x1B, 0x01])


class BedFormatError(ValueError):
    pass


@dataclass
class Genotypes:
    """Packed genotypes of I individuals x J SNPs (the SnpLinAlg role, loops.jl:527)."""
    data: np.ndarray   # uint8 (J, ceil(I/4)), C-contiguous
    I: int
    J: int

    @property
    def Ib(self) -> int:
        return (self.I + 3) // 4

    def __post_init__(self):
        if self.data.dtype != np.uint8 or self.data.shape != (self.J, self.Ib):
            raise BedFormatError(f"genotype bytes must be uint8 ({self.J}, {self.Ib}), got "
                                 f"{self.data.dtype} {self.data.shape}")
        self.data = np.ascontiguousarray(self.data)

    def decode(self) -> tuple[np.ndarray, np.ndarray]:
        """(g, nonmissing) as float64 arrays of shape (I, J), per loops.jl:2-5 (small cohorts)."""
        codes = np.empty((self.J, 4 * self.Ib), dtype=np.uint8)
        for s in range(4):
            codes[:, s::4] = (self.data >> (2 * s)) & 3
        codes = codes[:, : self.I].T
        gmap = np.array([0.0, 0.0, 1.0, 2.0])
        nmap = np.array([1.0, 0.0, 1.0, 1.0])
        return gmap[codes], nmap[codes]


def _count_lines(p: Path) -> int:
    with open(p, "rb") as f:
        return sum(1 for line in f if line.strip())


def read_bed(path: str | os.PathLike, I: int | None = None, J: int | None = None,
             mmap: bool = True) -> Genotypes:
    """Open a SNP-major .bed.  I/J default to the .fam/.bim line counts beside it."""
    path = Path(path)
    if path.suffix != ".bed":
        raise BedFormatError("filename should end with .bed")   # driver.jl:54
    stem = path.with_suffix("")
    if I is None:
        fam = stem.with_suffix(".fam")
        if not fam.exists():
            raise BedFormatError(f"{fam} not found and I not given")
        I = _count_lines(fam)
    if J is None:
        bim = stem.with_suffix(".bim")
        if not bim.exists():
            raise BedFormatError(f"{bim} not found and J not given")
        J = _count_lines(bim)
    Ib = (I + 3) // 4
    size = path.stat().st_size
    with open(path, "rb") as f:
        magic = f.read(3)
    if magic != BED_MAGIC:
        raise BedFormatError(f"{path}: bad magic {magic.hex()} (expected 6c1b01, SNP-major)")
    if size != 3 + Ib * J:
        raise BedFormatError(f"{path}: size {size} != 3 + {Ib} * {J} for I={I}, J={J}")
    if mmap:
        data = np.memmap(path, dtype=np.uint8, mode="r", offset=3, shape=(J, Ib))
        data = np.asarray(data)
    else:
        with open(path, "rb") as f:
            f.seek(3)
            data = np.frombuffer(f.read(), dtype=np.uint8).reshape(J, Ib).copy()
    return Genotypes(np.ascontiguousarray(data), I, J)


def write_bed(path: str | os.PathLike, g: Genotypes, write_sidecars: bool = True) -> Path:
    """Write magic + column bytes, and .bim/.fam with placeholder identifiers."""
    path = Path(path)
    with open(path, "wb") as f:
        f.write(BED_MAGIC)
        f.write(np.ascontiguousarray(g.data).tobytes())
    if write_sidecars:
        stem = path.with_suffix("")
        with open(stem.with_suffix(".fam"), "w") as f:
            for i in range(g.I):
                f.write(f"fam{i} ind{i} 0 0 0 -9\n")
        with open(stem.with_suffix(".bim"), "w") as f:
            for j in range(g.J):
                f.write(f"1 snp{j} 0 {j + 1} A C\n")
    return path


@dataclass
class DeviceGenotypes:
    """Packed genotypes already in device memory (the reference's g_cu, cuda/structs.jl:36-37):
    `data` is a CUDA tensor of uint8, shape (J, ceil(I/4)), one SNP column per row."""
    data: object
    I: int
    J: int

    @property
    def Ib(self) -> int:
        return (self.I + 3) // 4

    def to_host(self) -> Genotypes:
        return Genotypes(self.data.cpu().numpy(), self.I, self.J)
