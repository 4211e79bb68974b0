"""B200-native SQS optimisation hot path with the API of ``sqsgenerator``.

``parse_config`` and ``optimize`` mirror ``sqsgenerator.parse_config`` / ``sqsgenerator.optimize``;
the optimisation loop runs in hand-written sm_100a CUDA kernels behind the C ABI declared in
``include/sqsgen_b200.h``. There is no CPU fallback for the loop.
"""
from .config import parse_config
from .core import (IterationMode, LogLevel, ParseError, ParseErrorCode, Prec, ShellRadiiDetection, SqsConfiguration,
                   SqsResult, SqsResultPack, SqsResultSplit, SqsStatistics, Structure, SublatticeMode)
from .io import dump_result_pack, load_result_pack
from .optimize import optimize, prepare
from .serve import Server

__all__ = [
    "parse_config", "optimize", "prepare", "load_result_pack", "dump_result_pack", "IterationMode", "LogLevel",
    "ParseError", "ParseErrorCode", "Prec",
    "ShellRadiiDetection", "SqsConfiguration", "SqsResult", "SqsResultPack", "SqsResultSplit", "SqsStatistics",
    "Structure", "SublatticeMode", "Server",
]
