"""Statistics export: the reference's StatsExporter family for the engine's Stats.

Replaces ``CreateStatsExporter`` (src/io/stats/stats_exporter_factory.cc:11-22), ``ConsoleStatsExporter``
(src/io/stats/console_stats_exporter.cc:10-58) and ``StatsExportConfig`` / ``StatsExportFormat``
(src/config/stats_export_config.h). The counters come from the device: ``GpuPlocBvh.Build`` fills the
construction fields, ``Intersect(..., count=True)`` the 64-bit node-visit and triangle-test counts, and
``trace_frame(..., stats=...)`` the ray-tracing fields.

The console text is the reference's line for line with one fix: its "Traversals per query" line divides the
intersection count by the query count (console_stats_exporter.cc:41-43); here it divides the traversal count.
The reference's CSV format throws "not implemented yet" (stats_exporter_factory.cc:16-17); here it writes a
header row and one row per exported Stats, to a file (appending, header only when the file is new or empty) or
to standard output.
"""
from __future__ import annotations

import csv
import enum
import io
import os
import sys
from dataclasses import dataclass, fields

import numpy as np

from .accel import AccelerationStats, RaytracingStats, Stats


class StatsExportFormat(enum.Enum):
    kConsole = "console"
    kCsv = "csv"


def parse_stats_export_format(s: str) -> StatsExportFormat:
    """ParseEnum<StatsExportFormat> (stats_export_config.h:12-17)."""
    for f in StatsExportFormat:
        if f.value == s:
            return f
    raise ValueError(f"Invalid StatsExportFormat: {s}")


@dataclass
class StatsExportConfig:
    stats_export_format: StatsExportFormat = StatsExportFormat.kConsole
    path: str | None = None  # CSV destination; None = standard output


def _g3(x) -> str:
    # {:.3} of std::format on a floating-point value: shortest general form with 3 significant digits
    return format(float(x), ".3g")


class StatsExporter:
    def ExportOne(self, stats_export_config: StatsExportConfig, stats: Stats) -> None:
        raise NotImplementedError

    def ExportAll(self, stats_export_config: StatsExportConfig, stats_all) -> None:
        for s in stats_all:
            self.ExportOne(stats_export_config, s)


class ConsoleStatsExporter(StatsExporter):
    def __init__(self, stream=None):
        self.stream = stream

    def text(self, stats: Stats) -> str:
        rt, ac = stats.rt_stats, stats.accel_stats
        f32 = np.float32
        avg_i = (f32(0.0) if ac.query_count == 0 or ac.intersection_count == 0
                 else f32(ac.intersection_count) / f32(ac.query_count))
        avg_t = (f32(0.0) if ac.query_count == 0 or ac.traversal_count == 0
                 else f32(ac.traversal_count) / f32(ac.query_count))
        lines = [
            "########################################",
            "#                                      #",
            "#              Statistics              #",
            "#                                      #",
            "########################################",
            "",
            "----------------------------------------",
            "               Ray tracing              ",
            "----------------------------------------",
            f" Ray tracing time:              {_g3(rt.raytracing_time)} s",
            f" Primary ray count:             {rt.primary_ray_count}",
            f" Secondary ray count:           {rt.secondary_ray_count}",
            f" Shadow ray count:              {rt.shadow_ray_count}",
            "",
            "----------------------------------------",
            "               Acceleration             ",
            "----------------------------------------",
            "# Construction:                         ",
            f" Build time:                    {_g3(ac.build_time)} ms",
            f" Node count:                    {ac.node_count}",
            f" Inner node count:              {ac.inner_node_count}",
            f" Leaf node count:               {ac.leaf_node_count}",
            f" Memory consumption:            {_g3(f32(ac.memory_consumption) / f32(1e3))} KB",
            "",
            "# Traversal:                             ",
            f" Query count:                   {ac.query_count}",
            f" Intersection count:            {ac.intersection_count}",
            f" Intersections per query (avg): {_g3(avg_i)}",
            f" Traversal count:               {ac.traversal_count}",
            f" Traversals per query:          {_g3(avg_t)}",
            "",
            "########################################",
        ]
        return "\n".join(lines) + "\n"

    def ExportOne(self, stats_export_config: StatsExportConfig, stats: Stats) -> None:
        out = self.stream or sys.stdout
        out.write(self.text(stats))
        out.flush()


CSV_COLUMNS = [f.name for f in fields(RaytracingStats)] + [f.name for f in fields(AccelerationStats)]


class CsvStatsExporter(StatsExporter):
    def __init__(self, stream=None):
        self.stream = stream

    @staticmethod
    def row(stats: Stats) -> list:
        return ([getattr(stats.rt_stats, c) for c in CSV_COLUMNS[:len(fields(RaytracingStats))]] +
                [getattr(stats.accel_stats, c) for c in CSV_COLUMNS[len(fields(RaytracingStats)):]])

    def ExportAll(self, stats_export_config: StatsExportConfig, stats_all) -> None:
        stats_all = list(stats_all)
        if self.stream is None and stats_export_config.path:
            new = not os.path.exists(stats_export_config.path) or os.path.getsize(stats_export_config.path) == 0
            with open(stats_export_config.path, "a", newline="") as f:
                self._write(f, stats_all, header=new)
        else:
            self._write(self.stream or sys.stdout, stats_all, header=True)

    def ExportOne(self, stats_export_config: StatsExportConfig, stats: Stats) -> None:
        self.ExportAll(stats_export_config, [stats])

    @staticmethod
    def _write(f, stats_all, header: bool) -> None:
        w = csv.writer(f, lineterminator="\n")
        if header:
            w.writerow(CSV_COLUMNS)
        for s in stats_all:
            w.writerow(CsvStatsExporter.row(s))
        f.flush()


def CreateStatsExporter(stats_export_config: StatsExportConfig) -> StatsExporter:
    """CreateStatsExporter (stats_exporter_factory.cc:11-22)."""
    fmt = stats_export_config.stats_export_format
    if fmt == StatsExportFormat.kConsole:
        return ConsoleStatsExporter()
    if fmt == StatsExportFormat.kCsv:
        return CsvStatsExporter()
    raise ValueError("Unknown StatExportFormat")


def read_stats_csv(path_or_text: str) -> list:
    """Stats rows back from a CSV written by CsvStatsExporter (a path, or the text itself)."""
    text = open(path_or_text).read() if os.path.exists(path_or_text) else path_or_text
    rows = list(csv.DictReader(io.StringIO(text)))
    out = []
    for r in rows:
        s = Stats()
        for f in fields(RaytracingStats):
            setattr(s.rt_stats, f.name, (float if f.type in (float, "float") else int)(r[f.name]))
        for f in fields(AccelerationStats):
            setattr(s.accel_stats, f.name, (float if f.type in (float, "float") else int)(r[f.name]))
        out.append(s)
    return out
