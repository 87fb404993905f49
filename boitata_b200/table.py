"""Columnar table of per-target results, the shape of the reference's `Table`
(crates/py/src/table.rs:174-560): named float columns of equal length, read
as numpy arrays, exchanged with pyarrow and pandas."""

import numpy as np

from .errors import InvalidInput


class Table:
    """Named columns of equal length; `table["name"]` is a numpy array."""

    def __init__(self, columns):
        cols = {str(k): np.asarray(v) for k, v in dict(columns).items()}
        rows = {len(v) for v in cols.values()}
        if len(rows) > 1:
            raise InvalidInput("table columns must have equal lengths")
        self._cols = cols
        self._rows = rows.pop() if rows else 0

    @property
    def num_rows(self):
        return self._rows

    @property
    def column_names(self):
        return list(self._cols)

    def __len__(self):
        return self._rows

    def __contains__(self, name):
        return name in self._cols

    def __getitem__(self, name):
        try:
            return self._cols[name]
        except KeyError:
            raise KeyError(f"no column {name!r}; columns are {self.column_names}") from None

    def with_column(self, name, values):
        cols = dict(self._cols)
        cols[name] = values
        return Table(cols)

    def filter(self, mask):
        mask = np.asarray(mask, dtype=bool)
        if mask.shape != (self._rows,):
            raise InvalidInput(f"mask: expected {self._rows} values, got {mask.shape}")
        return Table({k: v[mask] for k, v in self._cols.items()})

    def to_pyarrow(self):
        import pyarrow as pa

        return pa.table(self._cols)

    def to_pandas(self):
        import pandas as pd

        return pd.DataFrame(self._cols)

    def __repr__(self):
        return f"Table({self._rows} rows: {', '.join(self.column_names)})"
