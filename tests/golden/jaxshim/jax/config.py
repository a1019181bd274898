"""``jax.config`` as a no-op store (test infrastructure)."""


class _Config:
    def __init__(self):
        self.values = {}

    def update(self, name, value):
        self.values[name] = value

    def __getattr__(self, name):
        return self.__dict__.get("values", {}).get(name, True)


config = _Config()
