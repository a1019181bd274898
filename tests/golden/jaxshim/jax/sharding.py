class Mesh:
    def __init__(self, *a, **k):
        raise NotImplementedError("sharding is outside the numpy stand-in")


NamedSharding = PartitionSpec = Mesh
